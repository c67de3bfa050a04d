"""Generate the instantiation units of the reference oracle library.

TEST INFRASTRUCTURE ONLY.  Writes oracle/_ref/gen/inst_*.cpp, each of which
instantiates a slice of the reference's filter logic types (through the
aliases in oracle/ref_bridge.hpp) and registers them by config.

  --set full   every config the reference's runtime dispatchers accept
               (blocked_bloomfilter.hpp:169-229, zoned_blocked_bloomfilter.hpp:
               174-215, cuckoofilter.hpp:184-206), both addressing modes
  --set bench  only the configs the benchmarks and the CPU baseline use
"""
import argparse
import os

BENCH_BLOOM = {(4, 1, 1, 1, 4), (8, 8, 8, 1, 8), (8, 8, 8, 2, 8), (8, 8, 8, 4, 8),
               (4, 16, 16, 2, 8), (4, 16, 16, 4, 8), (4, 1, 1, 1, 8)}
BENCH_CUCKOO = {(16, 4), (8, 4), (12, 4)}


def bloom_configs():
    out = []
    for wb in (4, 8):
        for w in (1, 2, 4, 8, 16):
            for s in (1, 2, 4, 8, 16):
                if s > w * wb:
                    continue
                for k in range(1, 17):
                    if k % s:
                        continue
                    out.append((wb, w, s, 1, k))
            if w >= 4:
                for z in (2, 4, 8):
                    if z >= w:
                        continue
                    for k in range(2, 17, 2):
                        if k % z:
                            continue
                        out.append((wb, w, w, z, k))
    return out


def cuckoo_configs():
    return [(t, b) for t in (4, 8, 12, 16, 32) for b in (1, 2, 4)]


ADDR = {0: "dtl::block_addressing::POWER_OF_TWO", 1: "dtl::block_addressing::MAGIC"}


def bloom_line(wb, w, s, z, k, a):
    tw = "uint32_t" if wb == 4 else "uint64_t"
    if z == 1:
        t = f"bbf_logic<{tw},{w},{s},{k},{ADDR[a]}>"
    else:
        t = f"zbbf_logic<{tw},{w},{z},{k},{ADDR[a]}>"
    return f"  register_bloom({{{wb},{w},{s},{z},{k},{a},&bloom_ops<{t}>::table}});"


def cuckoo_line(t, b, a):
    ty = f"cf_logic<{t},{b},{ADDR[a]}>"
    return f"  register_cuckoo({{{t},{b},0,0,0,{a},&cuckoo_ops<{ty}>::table}});"


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--set", choices=("full", "bench"), default="full")
    ap.add_argument("--out", required=True)
    ap.add_argument("--units", type=int, default=24)
    args = ap.parse_args()

    lines = []
    for c in bloom_configs():
        if args.set == "bench" and c not in BENCH_BLOOM:
            continue
        for a in (0, 1):
            lines.append(bloom_line(*c, a))
    for c in cuckoo_configs():
        if args.set == "bench" and c not in BENCH_CUCKOO:
            continue
        for a in (0, 1):
            lines.append(cuckoo_line(*c, a))

    os.makedirs(args.out, exist_ok=True)
    units = max(1, min(args.units, len(lines)))
    for u in range(units):
        chunk = lines[u::units]
        with open(os.path.join(args.out, f"inst_{u:02d}.cpp"), "w") as f:
            f.write("// generated by oracle/gen_ref_instances.py -- do not edit\n")
            f.write('#include "ref_bridge.hpp"\nnamespace refbridge {\n')
            f.write(f"struct reg_{u} {{ reg_{u}() {{\n")
            f.write("\n".join(chunk) + "\n")
            f.write(f"}} }} static reg_{u}_instance;\n}}\n")
    print(f"{len(lines)} instances in {units} units -> {args.out}")


if __name__ == "__main__":
    main()
