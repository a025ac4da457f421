#!/usr/bin/env python
"""Generate the golden vectors in tests/golden/ from the reference's own CPU code.

Runs oracle/_ref/kpz_ref (built by oracle/build_ref.py from the CudaKpz sources) and
stores its outputs as small fixtures.  Inputs that are random lattices are produced by the
oracle and stored alongside, so the fixtures stand alone.  Re-run after rebuilding the
reference binary:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import hashlib
import json
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))
from oracle import oracle as o  # noqa: E402

REF = ROOT / "oracle" / "_ref" / "kpz_ref"


def run(*args) -> list[str]:
    r = subprocess.run([str(REF), *map(str, args)], capture_output=True, text=True, check=True)
    return [ln for ln in r.stdout.splitlines() if ln and not ln.startswith("#")]


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.uint32).tobytes()).hexdigest()


def main():
    tmp = Path(tempfile.mkdtemp())
    # 1. C1: random-sequential CPU scheduler, 256^2, p=1 q=0, supplySeed(1,1), W^2 at 2^k
    ts = [1, 2, 4, 8, 16, 32, 64, 128, 256, 512]
    lines = run("rs", 8, 1, *ts, tmp / "rs.bin")
    rows = [[float(v) for v in ln.split()[1:]] for ln in lines]
    lat = np.fromfile(tmp / "rs.bin", dtype=np.uint32)
    (HERE / "ref_rs256_seed1.json").write_text(json.dumps(
        {"lx": 8, "seed": 1, "t": ts, "roughness": rows, "final_lattice_sha256": sha(lat),
         "source": "SchedulerCPU::mcs, kpz/schedulerCPU.cpp:35-38"}, indent=1))

    # 2. dSFMT-19937 draws
    d = {"seed1234_first8": [float(x) for x in run("dsfmt", 1234, 8)],
         "seed1_reseeded_first8": [float(x) for x in run("dsfmt", 1, 8, "reseed")]}
    (HERE / "ref_dsfmt.json").write_text(json.dumps(d, indent=1))

    # 3. deterministic SCA (p or q = 1): SchedulerCPUCBBit (ENC_CBBIT) and SchedulerCPUCB (ENC_LOCAL)
    cases = {}
    for lx in (6, 7, 8):
        for (p, q) in ((1.0, 0.0), (1.0, 1.0), (0.0, 1.0)):
            for init in ("flat", "rand"):
                for enc, cmd in ((1, "cbbit"), (0, "cb")):
                    if init == "flat":
                        w = o.homogeneous(lx, lx, enc)
                        src = "flat"
                    else:
                        w = o.random_lattice(lx, lx, o.ENC_CBBIT, seed=lx, mcs=5)
                        if enc == 0:
                            w = o.cbbit_to_local(w, lx, lx)
                        w.tofile(tmp / "in.bin")
                        src = tmp / "in.bin"
                    run(cmd, lx, p, q, 7, src, tmp / "out.bin", 1)
                    out = np.fromfile(tmp / "out.bin", dtype=np.uint32)
                    key = f"{cmd}_lx{lx}_p{p}_q{q}_{init}"
                    cases[key + "_in"] = w
                    cases[key + "_out"] = out
    np.savez_compressed(HERE / "ref_sca_deterministic.npz", **cases)

    # 4. roughness, correlator and consistency check on rough lattices
    an = {}
    for enc in (0, 1):
        for lx in (6, 8, 9):
            w = o.random_lattice(lx, lx, o.ENC_CBBIT, seed=3 + lx, mcs=9, p=0.6, q=0.3)
            s = o.random_lattice(lx, lx, o.ENC_CBBIT, seed=30 + lx, mcs=12, p=0.7, q=0.2)
            if enc == 0:
                w, s = o.cbbit_to_local(w, lx, lx), o.cbbit_to_local(s, lx, lx)
            w.tofile(tmp / "a.bin")
            s.tofile(tmp / "b.bin")
            key = f"enc{enc}_lx{lx}"
            an[key + "_sys"] = w
            an[key + "_snap"] = s
            an[key + "_rough"] = np.array(run("rough", enc, lx, tmp / "a.bin")[0].split(), dtype=float)
            an[key + "_corr"] = np.array(run("corr", enc, lx, tmp / "b.bin", tmp / "a.bin")[0].split(),
                                         dtype=float)
            if enc == 0:
                bad = w.copy()
                bad[3] ^= 1 << 4
                bad.tofile(tmp / "c.bin")
                an[key + "_check_valid"] = np.array(int(run("check", enc, lx, tmp / "a.bin")[0]))
                an[key + "_check_broken"] = np.array(int(run("check", enc, lx, tmp / "c.bin")[0]))
    np.savez_compressed(HERE / "ref_analysis.npz", **an)

    # 5. quenched binary disorder: generateDisorder2(0.3) then SchedulerCPU::mcsDisorder2(20)
    #    with class rates (p0,q0) = (0.9,0.1), (p1,q1) = (0.3,0.6); 256^2, seed 3
    run("rsdis", 8, 3, 0.3, 20, 0.9, 0.1, 0.3, 0.6, tmp / "dis.bin", tmp / "lat.bin")
    np.savez_compressed(HERE / "ref_disorder.npz",
                        disorder=np.fromfile(tmp / "dis.bin", dtype=np.uint32),
                        lattice=np.fromfile(tmp / "lat.bin", dtype=np.uint32))

    # 6. SchedulerService::saveBit file of the RS lattice (256^2, seed 1, 16 MCS): the lattice
    #    file format the checkpoint entry points keep (kpz/schedulerService.cpp:389-401)
    run("savebit", 8, 1, 16, HERE / "ref_savebit_rs256.bin", "CudaKpz saveBit fixture")
    inject_cases(tmp)
    print("golden vectors written to", HERE)


# rates, lx, MCS, start: random rates through the reference's per-site path
INJECT_CASES = [((0.5, 0.5), 8, 3, "flat"), ((0.9, 0.1), 9, 4, "flat"), ((0.3, 0.7), 8, 3, "rand"),
                ((0.75, 0.25), 8, 5, "rand"), ((0.95, 0.05), 9, 2, "flat")]
INJECT_SEED, INJECT_STREAM = 42, 3


def inject_cases(tmp: Path):
    """7. random rates: the reference's SchedulerCPUCBBit::mcsPQSyncRng per-site path
    (kpz/schedulerCPUCBBit_nested.inl:261-295) with its generator replaced by a stand-in that
    hands it the counter stream's per-site decisions (oracle/ref_inject.cpp), one thread;
    random starts are oracle lattices stored beside the results."""
    out = {}
    for (p, q), lx, n, init in INJECT_CASES:
        w = o.homogeneous(lx, lx, o.ENC_CBBIT) if init == "flat" else o.random_lattice(lx, lx, o.ENC_CBBIT, seed=8, mcs=3)
        key = f"p{p}_q{q}_lx{lx}_n{n}_{init}"
        w.tofile(tmp / "in.bin")
        run("cbbit-inject", lx, p, q, n, tmp / "in.bin", tmp / "out.bin", INJECT_SEED, INJECT_STREAM)
        if init != "flat":
            out[key + "_in"] = w
        out[key + "_out"] = np.fromfile(tmp / "out.bin", dtype=np.uint32)
    np.savez_compressed(HERE / "ref_inject_cbbit.npz", **out)


if __name__ == "__main__":
    if sys.argv[1:] == ["inject"]:
        inject_cases(Path(tempfile.mkdtemp()))
    else:
        main()
