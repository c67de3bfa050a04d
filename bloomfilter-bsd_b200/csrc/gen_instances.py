"""Writes the kernel instantiation units of libdtlg.so (build step).

Every Bloom config the reference's runtime dispatchers accept
(blocked_bloomfilter.hpp:169-229, zoned_blocked_bloomfilter.hpp:174-215) gets
a compiled probe and build kernel; the units are spread so nvcc can compile
them in parallel.  Output: <out>/bloom_inst_NN.cu
"""
import argparse
import os


def bloom_configs():
    out = []
    for wb in (4, 8):
        for w in (1, 2, 4, 8, 16):
            for s in (1, 2, 4, 8, 16):
                if s > w * wb:
                    continue
                for k in range(1, 17):
                    if k % s == 0:
                        out.append((wb, w, s, 1, k))
            if w >= 4:
                for z in (2, 4, 8):
                    if z < w:
                        for k in range(2, 17, 2):
                            if k % z == 0:
                                out.append((wb, w, w, z, k))
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    ap.add_argument("--units", type=int, default=16)
    args = ap.parse_args()
    cfgs = bloom_configs()
    os.makedirs(args.out, exist_ok=True)
    for u in range(args.units):
        lines = []
        for (wb, w, s, z, k) in cfgs[u::args.units]:
            word = "uint32_t" if wb == 4 else "uint64_t"
            lines.append(f"  register_bloom(bloom_entry<{word}, {w}, {s}, {z}, {k}>());")
        body = ("// generated by csrc/gen_instances.py\n#include \"registry.hpp\"\n"
                "namespace dtlg {\nnamespace {\n"
                f"struct Reg{u} {{\n  Reg{u}() {{\n" + "\n".join(lines) + f"\n  }}\n}} reg{u};\n"
                "}  // namespace\n}  // namespace dtlg\n")
        path = os.path.join(args.out, f"bloom_inst_{u:02d}.cu")
        old = open(path).read() if os.path.exists(path) else None
        if old != body:
            with open(path, "w") as f:
                f.write(body)
    print(f"{len(cfgs)} bloom configs in {args.units} units")


if __name__ == "__main__":
    main()
