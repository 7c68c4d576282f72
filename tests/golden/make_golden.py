"""Generates the golden fixtures in this directory (run once, on the CPU).

Each fixture pins one workload: the generator's output (sha256 of the CSR) and
the oracle's truss decomposition of it (sha256 of the truss numbers as u32
little-endian per CSR slot, their histogram, triangle count, k_max).  Small
graphs also store the full truss arrays.  The oracle used per workload is
recorded: the restatement of the reference's PKT (oracle.pkt) wherever it
finishes in minutes, cross-checked against the restated Burkhardt peel and
the independent exact peel (oracle.fast_truss); the independent peel alone for
R-MAT-22 and R-MAT-24, where the restatement's hash-map-per-frontier-edge
processing would take hours.

Every mode-0 fixture is also certified by the corrected verifier
(oracle.verify: symmetric truss, support >= k - 2 inside the k-truss, local
maximality), an independent check of the truss definition that does not
depend on any peel; ``"verified": true`` records a pass.  ``--verify`` runs
that certification alone on fixtures already in the file (regenerating each
graph and its truss, which must hash to the stored values).

    python tests/golden/make_golden.py [--only NAME ...] [--verify]
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from sparkx_b200 import gen  # noqa: E402

# (name, generator kwargs, oracle modes)
WORKLOADS = {
    "cfg1_er_100k_1m": dict(fn="er", n=100_000, m=1_000_000, seed=1, oracles=("pkt", "burkhardt", "fast"),
                            modes=(0, 1)),
    "cfg2_rmat22": dict(fn="rmat", scale=22, ef=16, seed=2, oracles=("fast", "pkt"), modes=(0,)),
    # config 5's 1% tail: the first R-MAT-24 request of the served stream
    "cfg5_rmat24_tail": dict(fn="rmat", scale=24, ef=16, seed=100, oracles=("fast",), modes=(0,)),
    "cfg3_debruijn": dict(fn="dbg", seq_len=20_000_000, k=21, copies=1000, seg_len=10_000, mut_rate=0.05,
                          seed=3, oracles=("pkt", "fast"), modes=(0, 1)),
    "rmat16": dict(fn="rmat", scale=16, ef=16, seed=2, oracles=("pkt", "burkhardt", "fast"), modes=(0, 1)),
    "rmat18": dict(fn="rmat", scale=18, ef=16, seed=2, oracles=("pkt", "fast"), modes=(0, 1)),
    # the PKT restatement against the independent peel one size above R-MAT-18
    "rmat20": dict(fn="rmat", scale=20, ef=16, seed=2, oracles=("pkt", "fast"), modes=(0,)),
    "dbg_small": dict(fn="dbg", seq_len=200_000, k=21, copies=50, seg_len=2_000, mut_rate=0.05, seed=3,
                      oracles=("pkt", "burkhardt", "fast"), modes=(0, 1)),
    # small graphs whose full truss arrays are committed
    "arr_rmat10": dict(fn="rmat", scale=10, ef=16, seed=21, oracles=("pkt", "burkhardt", "fast"), modes=(0, 1),
                       arrays=True),
    "arr_dbg_k6": dict(fn="dbg", seq_len=3_000, k=6, copies=8, seg_len=200, mut_rate=0.05, seed=22,
                       oracles=("pkt", "burkhardt", "fast"), modes=(0,), arrays=True),
    "arr_er": dict(fn="er", n=2_000, m=20_000, seed=23, oracles=("pkt", "burkhardt", "fast"), modes=(0,),
                   arrays=True),
}
MIX_MEMBERS = 24  # first members of the batched mix (config 4) with n <= 2e5


def graph_for(spec):
    if spec["fn"] == "er":
        return gen.erdos_renyi(spec["n"], spec["m"], spec["seed"])
    if spec["fn"] == "rmat":
        return gen.rmat(spec["scale"], spec["ef"], seed=spec["seed"])
    if spec["fn"] == "dbg":
        return gen.debruijn(spec["seq_len"], spec["k"], spec["copies"], spec["seg_len"], spec["mut_rate"],
                            spec["seed"])
    if spec["fn"] == "mix":
        return gen.mix_graph(gen.mix_member(spec["index"]))
    raise ValueError(spec)


def csr_sha(g) -> str:
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(g.offsets, dtype="<u8").tobytes())
    h.update(np.ascontiguousarray(g.neighbours, dtype="<u4").tobytes())
    return h.hexdigest()


def truss_sha(t) -> str:
    return hashlib.sha256(np.ascontiguousarray(t, dtype="<u4").tobytes()).hexdigest()


def run_oracle(name, g, mode):
    if name == "pkt":
        return O.pkt(g.offsets, g.neighbours, mode=mode, threads=os.cpu_count() or 1)
    if name == "burkhardt":
        return O.burkhardt(g.offsets, g.neighbours, mode=mode)
    if name == "fast":
        return O.fast_truss(g.offsets, g.neighbours, mode=mode)[0]
    raise ValueError(name)


def fixture(name, spec):
    t0 = time.time()
    g = graph_for(spec)
    sup = None
    out = {"name": name, "params": {k: v for k, v in spec.items() if k not in ("oracles", "modes", "arrays")},
           "csr_sha256": csr_sha(g), "n": g.n, "width": g.width, "modes": {}}
    for mode in spec.get("modes", (0,)):
        results = {}
        # with u8 counters the reference's Burkhardt peel (a count that wraps to
        # 0 reads as a removed edge) and its PKT peel (counts clamp at the
        # level) legitimately differ; the drop-in target is AlgoPKT, so u8
        # fixtures pin the PKT restatement
        for o in spec["oracles"]:
            if mode == 1 and o == "burkhardt":
                continue
            try:
                results[o] = run_oracle(o, g, mode)
            except O.OracleError as e:
                results[o] = str(e)
        base = next(iter(results.values()))
        agree = all(isinstance(v, np.ndarray) and np.array_equal(v, base) for v in results.values())
        if isinstance(base, str):
            out["modes"][str(mode)] = {"error": base, "oracles": list(results)}
            continue
        if not agree:
            raise SystemExit(f"{name} mode {mode}: oracles disagree")
        if mode == 0:
            _, tri, _ = O.fast_truss(g.offsets, g.neighbours)
            out["triangles"] = tri
        hist = np.bincount(base.astype(np.int64))
        out["modes"][str(mode)] = {"truss_sha256": truss_sha(base), "k_max": int(base.max()) if base.size else 0,
                                   "hist": {str(i): int(c) for i, c in enumerate(hist) if c},
                                   "oracles": list(results)}
        if mode == 0:
            out["modes"]["0"].update(certify(g, base))
        if spec.get("arrays"):
            arr = os.path.join(HERE, f"{name}.npz")
            prev = dict(np.load(arr)) if mode and os.path.exists(arr) else {}
            prev.update({"offsets": g.offsets, "neighbours": g.neighbours, f"truss_mode{mode}": base.astype(np.uint32)})
            if mode == 0:
                prev["brute_force"] = O.brute_force_truss(g.offsets, g.neighbours) if g.width < 30_000 else base
            np.savez_compressed(arr, **prev)
    out["seconds"] = round(time.time() - t0, 1)
    print(name, out["seconds"], "s", flush=True)
    return out


def certify(g, truss):
    """The corrected verifier's verdict on a truss assignment (mode 0 only: the
    u8 mode's wrapped counts are not a truss decomposition)."""
    t0 = time.time()
    bad = O.verify(g.offsets, g.neighbours, truss, threads=os.cpu_count() or 1)
    if bad >= 0:
        raise SystemExit(f"verifier rejects slot {bad}")
    return {"verified": True, "verify_seconds": round(time.time() - t0, 1)}


def verify_existing(name, entry):
    """Regenerate a stored fixture's graph and truss, check both hashes, certify."""
    spec = WORKLOADS.get(name)
    if spec is None and name.startswith("cfg4_mix_"):
        spec = dict(fn="mix", index=int(name.rsplit("_", 1)[1]))
    g = graph_for(spec)
    if csr_sha(g) != entry["csr_sha256"]:
        raise SystemExit(f"{name}: generator output changed")
    truss = O.fast_truss(g.offsets, g.neighbours)[0]
    if truss_sha(truss) != entry["modes"]["0"]["truss_sha256"]:
        raise SystemExit(f"{name}: truss differs from the stored fixture")
    res = certify(g, truss)
    print(name, "verified in", res["verify_seconds"], "s", flush=True)
    return res


def mix_fixtures():
    res = []
    i = 0
    while len(res) < MIX_MEMBERS:
        mem = gen.mix_member(i)
        if mem.n <= 200_000:
            spec = dict(fn="mix", index=i, oracles=("pkt", "fast"), modes=(0,))
            f = fixture(f"cfg4_mix_{i}", spec)
            f["member"] = {"kind": mem.kind, "n": mem.n, "pairs": mem.pairs, "avg_degree": mem.avg_degree,
                           "seed": mem.seed}
            res.append(f)
        i += 1
    return res


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--only", nargs="*")
    ap.add_argument("--verify", action="store_true", help="certify stored fixtures only")
    args = ap.parse_args()
    O.build()
    path = os.path.join(HERE, "fixtures.json")
    data = {}
    if os.path.exists(path):
        with open(path) as f:
            data = json.load(f)
    if args.verify:
        for name in args.only or sorted(data):
            res = verify_existing(name, data[name])
            with open(path) as f:
                current = json.load(f)
            current[name]["modes"]["0"].update(res)
            with open(path, "w") as f:
                json.dump(current, f, indent=1, sort_keys=True)
        return
    names = args.only or list(WORKLOADS) + ["cfg4_mix"]
    for name in names:
        if name == "cfg4_mix":
            for f in mix_fixtures():
                data[f["name"]] = f
        else:
            data[name] = fixture(name, WORKLOADS[name])
        # merge with the file as it is now (another run may have added entries)
        current = {}
        if os.path.exists(path):
            with open(path) as f:
                current = json.load(f)
        current.update({k: v for k, v in data.items()})
        data = current
        with open(path, "w") as f:
            json.dump(data, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
