"""GPU calibrations in the reference's calibration-data file format.

The reference keeps its calibration in a binary file (format version 1,
model/calibration_data.cpp:144-330, read by calibration_data::open_file): a
PNG-like signature, the memory levels with their cache sizes and reference
filter sizes, per Bloom and cuckoo configuration one lookup-cost delta per
memory level plus tuning parameters, and the skyline matrix
(model/skyline_matrix.hpp:22-162).  Writing GPU calibrations in that format
lets the reference's own tools read them: its skyline lookup behind
filter::construct(n, tw, ...) and its cost model cost_fn::lookup_costs.

The reference's model prices a lookup as sum_l dt_l * p_miss(l-1, m) with
p_miss(l, m) = 1 - cache_l / m beyond the cache (cost_fn.hpp:39-48,127-141).
For a GPU the levels are L2 and HBM: dt_1 = the calibrated time of a filter
well inside L2, dt_2 = (t(m_2) - dt_1) / p_miss(1, m_2) for a filter far
beyond it (compute_delta_tls, cost_fn.hpp:80-123).  Times are per lookup in
the GPU's aggregate throughput terms (ns per key), cycles at the SM clock.

Units: the reference's calibration stores cache sizes in bits
(calibration.cpp:98-101), but its query-time lookup cost compares them with
the filter size in BYTES (cost_fn.hpp:135-139: m / 8).  The file holds the L2
size in bytes, the unit that lookup reads, so that the reference prices a GPU
filter of m bits by the cost measured for it; the reference filter sizes are
in bits, as the reference writes them.

Layout (little endian): signature, u64 version, u64 mem levels L, (L-1) u64
cache sizes [bits], L u64 filter sizes [bits], u64 #bloom configs, u64 #cuckoo
configs, bloom configs (6 x u32: k, word size, words per block, sectors,
addressing, zones), their L timings (2 x f64: cycles, ns), their tuning
parameters (u32 unroll factor), the same for cuckoo configs (3 x u32: tag
bits, tags per bucket, addressing), then the skyline matrix: u64 #n, u64 #tw,
the n and tw values (u64), and #n x #tw entries (config, u64 m, timing) at
index tw_idx * #n + n_idx.
"""
import struct

import numpy as np

from . import cost as CM

SIGNATURE = bytes([0o211]) + b"FIL\r\n" + bytes([0o32]) + b"\n"
VERSION = 1
POW2, MAGIC = 0, 1


def _bloom_key(c, addr):
    return (c.k, c.word_size, c.w, c.s, addr, c.z)


def _interp_ns(calib, ci, log2_bytes):
    return float(np.interp(log2_bytes, calib.log2_bytes, calib.ns_per_key[ci]))


def delta_tls(t_l2, t_hbm, cache, m_l2, m_hbm):
    """compute_delta_tls (cost_fn.hpp:80-123) for the two GPU levels (sizes in one unit)."""
    assert m_l2 <= cache < m_hbm
    p = 1.0 - cache / m_hbm
    return t_l2, (t_hbm - t_l2) / p


def write_reference_file(path, model: CM.CostModel, l2_bytes=126 << 20, clock_ghz=1.965,
                         n_log2=range(10, 25), tw_log2=range(4, 25)):
    """Writes `model`'s calibration (and a skyline matrix built by its
    exhaustive search over the Bloom candidates) as a reference file."""
    calib = model.calib
    cache = int(l2_bytes)                    # bytes: the unit of the reference's lookup (see above)
    m_l2 = (int(l2_bytes) // 4) * 8          # a filter a quarter of the L2 size [bits]
    m_hbm = (1 << 30) * 8                    # a 1 GiB filter [bits]
    sizes = [m_l2, m_hbm]

    def timings(ci):
        d1, d2 = delta_tls(_interp_ns(calib, ci, np.log2(m_l2 / 8)), _interp_ns(calib, ci, np.log2(m_hbm / 8)),
                           cache, m_l2 // 8, m_hbm // 8)
        return [(d * clock_ghz, d) for d in (d1, d2)]

    blooms, cuckoos = [], []
    for ci, c in enumerate(calib.candidates):
        for addr in (POW2, MAGIC):
            if c.kind == "bloom":
                blooms.append((_bloom_key(c, addr), timings(ci)))
            else:
                cuckoos.append(((c.t, c.b, addr), timings(ci)))
    blooms.sort(key=lambda x: x[0])
    cuckoos.sort(key=lambda x: x[0])

    out = bytearray(SIGNATURE)
    out += struct.pack("<QQ", VERSION, 2)
    out += struct.pack("<Q", cache)
    out += struct.pack("<2Q", *sizes)
    out += struct.pack("<QQ", len(blooms), len(cuckoos))
    for key, _ in blooms:
        out += struct.pack("<6I", *key)
    for _, ts in blooms:
        for cyc, ns in ts:
            out += struct.pack("<2d", cyc, ns)
    out += struct.pack(f"<{len(blooms)}I", *([1] * len(blooms)))
    for key, _ in cuckoos:
        out += struct.pack("<3I", *key)
    for _, ts in cuckoos:
        for cyc, ns in ts:
            out += struct.pack("<2d", cyc, ns)
    out += struct.pack(f"<{len(cuckoos)}I", *([1] * len(cuckoos)))

    # skyline: the best Bloom configuration and size per (n, tw) grid point
    n_vals = [1 << int(e) for e in n_log2]
    tw_vals = [1 << int(e) for e in tw_log2]
    bloom_idx = np.array([i for i, c in enumerate(calib.candidates) if c.kind == "bloom"])
    entries = []
    for tw in tw_vals:
        q = CM.make_queries(np.log2(n_vals), 1.0, 0.0, tw / clock_ghz, 0)
        r = model.search(q, per_candidate=True)
        for j, n in enumerate(n_vals):
            costs = r["cand_cost"][j, bloom_idx]
            b = int(bloom_idx[int(np.argmin(costs))])
            bpk = float(r["cand_bpk"][j, b])
            c = calib.candidates[b]
            entries.append((_bloom_key(c, MAGIC), int(round(bpk * n)), float(costs.min())))
    out += struct.pack("<QQ", len(n_vals), len(tw_vals))
    out += struct.pack(f"<{len(n_vals)}Q", *n_vals)
    out += struct.pack(f"<{len(tw_vals)}Q", *tw_vals)
    for key, m, ns in entries:
        out += struct.pack("<6IQ2d", *key, m, ns * clock_ghz, ns)
    with open(path, "wb") as f:
        f.write(out)
    return {"bloom_configs": len(blooms), "cuckoo_configs": len(cuckoos), "skyline": (len(n_vals), len(tw_vals)),
            "bytes": len(out)}


def read_reference_file(path):
    """Parses a reference calibration file (any memory-level count)."""
    b = open(path, "rb").read()
    if b[:8] != SIGNATURE:
        raise ValueError("not a calibration-data file")
    version, L = struct.unpack_from("<QQ", b, 8)
    if version != VERSION:
        raise ValueError(f"version {version}")
    o = 24
    caches = list(struct.unpack_from(f"<{L - 1}Q", b, o))
    o += 8 * (L - 1)
    sizes = list(struct.unpack_from(f"<{L}Q", b, o))
    o += 8 * L
    nb, nc = struct.unpack_from("<QQ", b, o)
    o += 16
    bkeys = [struct.unpack_from("<6I", b, o + 24 * i) for i in range(nb)]
    o += 24 * nb
    bt = np.frombuffer(b, dtype="<f8", count=nb * L * 2, offset=o).reshape(nb, L, 2)
    o += 16 * L * nb + 4 * nb
    ckeys = [struct.unpack_from("<3I", b, o + 12 * i) for i in range(nc)]
    o += 12 * nc
    ct = np.frombuffer(b, dtype="<f8", count=nc * L * 2, offset=o).reshape(nc, L, 2)
    o += 16 * L * nc + 4 * nc
    out = {"mem_levels": L, "cache_sizes": caches, "filter_sizes": sizes, "bloom": dict(zip(bkeys, bt)),
           "cuckoo": dict(zip(ckeys, ct)), "skyline": None}
    if o < len(b):
        n_cnt, tw_cnt = struct.unpack_from("<QQ", b, o)
        o += 16
        n_vals = struct.unpack_from(f"<{n_cnt}Q", b, o)
        o += 8 * n_cnt
        tw_vals = struct.unpack_from(f"<{tw_cnt}Q", b, o)
        o += 8 * tw_cnt
        ent = [struct.unpack_from("<6IQ2d", b, o + 48 * i) for i in range(n_cnt * tw_cnt)]
        out["skyline"] = {"n": list(n_vals), "tw": list(tw_vals), "entries": ent}
    return out


def main():
    import argparse
    import json
    import os

    from .calibration import CalibrationData
    ap = argparse.ArgumentParser(description="Write the packaged GPU calibration as the reference's "
                                             "calibration-data file (its default location is ~/.dtl-filter.dat).")
    ap.add_argument("--out", default=os.path.join(os.path.expanduser("~"), ".dtl-filter.dat"))
    ap.add_argument("--calibration", default=None)
    ap.add_argument("--l2-bytes", type=int, default=126 << 20)
    ap.add_argument("--clock-ghz", type=float, default=1.965)
    args = ap.parse_args()
    calib = CalibrationData.load(args.calibration) if args.calibration else CalibrationData.load()
    info = write_reference_file(args.out, CM.CostModel(calib), args.l2_bytes, args.clock_ghz)
    print(json.dumps({"out": args.out, **info}))


if __name__ == "__main__":
    main()
