#!/usr/bin/env python
"""Build the reference's own CPU schedulers into oracle/_ref/kpz_ref -- TEST INFRASTRUCTURE.

Compiles CudaKpz sources where they lie (read from the tree named by KPZ_REFERENCE, by default
the `reference` directory beside this repository; never copied into this
repository) together with oracle/ref_driver.cpp.  The reference's own build system needs
MPI, HDF5/libSplash and a TinyMT parameter table that is not shipped, and its code falls off
the end of several non-void functions, which current g++ turns into traps.  So this recipe:

  1. copies kpz/ and inc/ to a scratch directory under /tmp (outside this repository),
  2. removes the HDF5/libSplash/MPI include lines and the I/O function bodies that need them
     (writeH5/readH5/collectH5/retrieveH5/mcsH5/closeH5/syncRNGMPI, Correlator::save/fromH5,
     SystemSize::splashDimensions) -- none is on the hot path,
  3. adds the missing return statements,
  4. writes a placeholder TinyMT parameter table (TinyMT's published default parameter set
     repeated; the reference's table is absent, so TinyMT streams are not the reference's),
  5. compiles with g++ -O2 and writes the binary to oracle/_ref/kpz_ref (with oracle/ref_inject.cpp,
     the reference's CBBit scheduler fed this project's per-site decisions, and the C oracle).

Only code paths that do not depend on the TinyMT table are used as golden vectors
(p = 1 or q = 1 deterministic SCA, dSFMT random-sequential, roughness, correlator).
"""
from __future__ import annotations

import os
import re
import shutil
import subprocess
import sys
from pathlib import Path

REF = Path(os.environ.get("KPZ_REFERENCE", str(Path(__file__).resolve().parent.parent.parent / "reference")))
HERE = Path(__file__).resolve().parent
OUT = HERE / "_ref"
WORK = Path("/tmp/kpzb_refbuild")

SOURCES = [
    "kpz/systemSize.cpp", "kpz/threadLayout.cpp", "kpz/roughness.cpp", "kpz/schedulerService.cpp",
    "kpz/schedulerServiceStash.cpp", "kpz/correlator.cpp", "kpz/correlatorLines.cpp",
    "kpz/schedulerCPU.cpp", "kpz/schedulerCPUBase.cpp", "kpz/schedulerCPUBaseThreaded.cpp",
    "kpz/CPURngIface.cpp", "kpz/schedulerCPUCBBit_instances.cpp", "kpz/schedulerCPUCB_instances.cpp",
    "kpz/schedulerCPUDTr_instances.cpp",
    "inc/dSFMT/dSFMT.cpp", "inc/tinyMT/tinymt32.c", "inc/timer.cpp",
]

STUB = """// forward declarations replacing the HDF5/libSplash/MPI headers (I/O is not built)
#pragma once
#include <string>
#include <sstream>
namespace splash { class DataCollector; class Dimensions; class Selection; }
namespace MPI { class Comm; }
"""


def cut_between(text: str, start: str, end: str | None) -> str:
    a = text.index(start)
    b = text.index(end, a) if end else len(text)
    return text[:a] + text[b:]


def add_return(text: str, signature: str, stmt: str) -> str:
    """Insert `stmt` before the closing brace of the function whose header starts with signature."""
    a = text.index(signature)
    i = text.index("{", a)
    depth = 0
    for j in range(i, len(text)):
        if text[j] == "{":
            depth += 1
        elif text[j] == "}":
            depth -= 1
            if depth == 0:
                return text[:j] + "\t" + stmt + "\n" + text[j:]
    raise ValueError(signature)


def patch(work: Path) -> None:
    for p in list(work.rglob("*.cpp")) + list(work.rglob("*.h")) + list(work.rglob("*.inl")):
        t = p.read_text(errors="replace")
        t2 = re.sub(r"#include\s*<(mpi\.h|splash/splash\.h|KMCsplash\.h)>", "", t)
        if t2 != t:
            p.write_text(t2)
    ss = work / "kpz/schedulerService.cpp"
    t = ss.read_text()
    t = cut_between(t, "splash::DataCollector* Kpz::SchedulerService::writeH5",
                    "void* Kpz::SchedulerService::callMcs")
    t = cut_between(t, "int Kpz::SchedulerService::syncRNGMPI", "void Kpz::SchedulerService::setMcs")
    ss.write_text(t)
    co = work / "kpz/correlator.cpp"
    t = co.read_text()
    t = cut_between(t, "void Kpz::Correlator::save", "std::ostream& operator<< (std::ostream& o, const Kpz::Correlator& c)")
    for fn in ("correlateThreadCO", "correlateThreadCBBit", "roughnessThreadCO", "roughnessThreadCBBit"):
        t = add_return(t, f"void* Kpz::Correlator::{fn}(void* cd)", "return 0;")
    co.write_text(t)
    sz = work / "kpz/systemSize.cpp"
    t = sz.read_text()
    t = cut_between(t, "splash::Dimensions Kpz::SystemSize::splashDimensions", None)
    t = add_return(t, "bool Kpz::SystemSizeBase::set(int lx, int ly)", "return true;")
    t = add_return(t, "std::ostream& Kpz::operator<<(std::ostream& o, const Kpz::SystemSize& s)", "return o;")
    sz.write_text(t)
    ro = work / "kpz/roughness.cpp"
    t = ro.read_text()
    t = add_return(t, "const Kpz::Roughness& Kpz::Roughness::operator+=", "return *this;")
    t = add_return(t, "const Kpz::Roughness& Kpz::Roughness::operator/=", "return *this;")
    ro.write_text(t)
    bt = work / "kpz/schedulerCPUBaseThreaded.cpp"
    t = bt.read_text()
    m = re.search(r"\n(\w[^\n]*joinAllWorkers\([^)]*\))", t)
    if m and not m.group(1).startswith("void"):
        t = add_return(t, m.group(1), "return 0;")
    bt.write_text(t)
    for hdr in ("kpz/schedulerCPUBaseThreaded.h", "kpz/schedulerCPUpThread.h"):
        p = work / hdr
        t = p.read_text()
        m = re.search(r"(static void\* func_mcs\([^)]*\))", t)
        if m:
            t = add_return(t, m.group(1), "return 0;")
        p.write_text(t)
    tmt = work / "inc/tinyMT/tinymt32_param.h"
    n = 4096
    tmt.write_text(
        "// placeholder TinyMT32 parameter table: TinyMT's published default set, repeated\n"
        f"#pragma once\n#define KMC_N_TMT_PARAM_SETS {n}\n"
        + "".join(f"static const unsigned int {name}[{n}] = {{" + ",".join([val] * n) + "};\n"
                  for name, val in (("tinyMTmat1", "0x8f7011eeu"), ("tinyMTmat2", "0xfc78ff1fu"),
                                    ("tinyMTtmat", "0x3793fdffu"))))
    (work / "stub_io.h").write_text(STUB)


GPU_SOURCES = [
    "kpz/schedulerGPU.cu", "kpz/schedulerBase.cu", "kpz/GPURandom.cu", "kpz/GPUTinyMT.cu",
    "kpz/kpzSCABit.cu", "kpz/schedulerSCABit.cu", "kpz/correlatorCuda.cu", "inc/kmcExceptCUDA.cu",
    "kpz/kpz.cu", "kpz/schedulerDT.cu", "kpz/scheduler.cu",
]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")


def patch_gpu(work: Path) -> None:
    """Prepare the CUDA sources: drop the libSplash include (the schedulers' RNG-state HDF5
    methods then only name the forward-declared splash::DataCollector), make TinyMT32's HDF5
    bodies no-ops, and -- because the non-Fermi build defines only the default and "dis" DT
    layouts, which are the same type (kpz/schedulerDT.h:45-46) -- instantiate SchedulerDT once
    per RNG instead of the Fermi list (kpz/schedulerDTInstances.h:30-44)."""
    for p in work.rglob("*.cu"):
        t = p.read_text(errors="replace")
        t2 = re.sub(r"#include\s*<KMCsplash\.h>", "", t)
        if t2 != t:
            p.write_text(t2)
    tmt = work / "kpz/GPUTinyMT.cu"
    t = tmt.read_text()
    t = cut_between(t, "void TinyMT32::writeH5", None)
    t += ("void TinyMT32::writeH5(splash::DataCollector*, int, const std::string&) {}\n"
          "bool TinyMT32::readH5(splash::DataCollector*, int, const std::string&) { return false; }\n")
    tmt.write_text(t)
    di = work / "kpz/schedulerDTInstances.h"
    t = di.read_text()
    a = t.index("\ttemplate class SchedulerDT<SLCG64, SchedulerDT_LocalLayoutDefault>;")
    b = t.index("}", a)
    t = (t[:a] + "\ttemplate class SchedulerDT<SLCG64, SchedulerDT_LocalLayoutDis>;\n"
         "\ttemplate class SchedulerDT<TinyMT32, SchedulerDT_LocalLayoutDis>;\n" + t[b:])
    di.write_text(t)
    # BaseDTInnerDBSHRep's warp reduction uses the pre-CUDA-9 __shfl_xor, which does not exist
    # for sm_70 and later; the full-warp __shfl_xor_sync is the same butterfly
    ib = work / "kpz/kpzSimulationPrimitivesTemplates_BaseInnerDB.cu"
    t = ib.read_text()
    ib.write_text(t.replace("__shfl_xor(borderHits, a, 32)", "__shfl_xor_sync(0xffffffffu, borderHits, a, 32)"))


def build_gpu(cpu_objs: list[str]) -> None:
    """The reference's GPU SchedulerSCABit<SLCG64> for sm_100a, as its own Makefile builds it
    (kpz/Makefile: -O3 -maxrregcount=32 -DMODE_CUDA), linked with oracle/ref_gpu_driver.cu into
    oracle/_ref/kpz_ref_gpu.  -DNDEBUG drops the host assert in SLCG64::randomize
    (kpz/GPURandom.cu:44), whose bound (30721 streams, kpz/kpzConst.h:85) is below the
    151552 streams the scheduler asks for on 148 SMs; no device code changes."""
    if not Path(NVCC).exists():
        print("nvcc not found; skipping the reference GPU build", file=sys.stderr)
        return
    patch_gpu(WORK)
    flags = ["-O3", "-std=c++14", "-w", "-gencode", "arch=compute_100a,code=sm_100a", "-maxrregcount=32",
             "-DMODE_CUDA", "-DNDEBUG", "-DDSFMT_MEXP=19937", "-DKPZ_SWITCH_RNG=SLCG64",
             f"-I{WORK / 'kpz'}", f"-I{WORK / 'inc'}", "-include", str(WORK / "stub_io.h"), "-Xcompiler", "-pthread"]
    objs = []
    for src in GPU_SOURCES:
        obj = WORK / (Path(src).stem + ".cu.o")
        subprocess.run([NVCC, *flags, "-c", str(WORK / src), "-o", str(obj)], check=True)
        objs.append(str(obj))
    drv = WORK / "ref_gpu_driver.o"
    subprocess.run([NVCC, *flags, "-c", str(HERE / "ref_gpu_driver.cu"), "-o", str(drv)], check=True)
    cpu = [o for o in cpu_objs if not o.endswith("ref_driver.o")]
    subprocess.run([NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-o", str(OUT / "kpz_ref_gpu"),
                    str(drv), *objs, *cpu, "-Xcompiler", "-pthread", "-lcudart"], check=True)
    print(f"built {OUT / 'kpz_ref_gpu'}")
    # further builds with the other inner schemes the DT kernel here implements: single-hit
    # double tiling (KPZ_INNER_DT), dead border (KPZ_INNER_DB), double tiling with a random cell
    # offset (KPZ_INNER_DTDBSH) and DBSH with replaced borders (KPZ_INNER_DBSHREP),
    # kpz/kpzConst.h:26-35
    param = WORK / "kpz/param.h"
    t = param.read_text()
    for tag, dd in (("innerdt", "KPZ_INNER_DT"), ("innerdb", "KPZ_INNER_DB"), ("innerdtdbsh", "KPZ_INNER_DTDBSH"),
                    ("innerdbshrep", "KPZ_INNER_DBSHREP")):
        param.write_text(t.replace("#define KPZ_INNER_DD KPZ_INNER_DBSH", f"#define KPZ_INNER_DD {dd}"))
        objs2 = []
        for src in GPU_SOURCES:
            obj = WORK / (Path(src).stem + f".{tag}.cu.o")
            subprocess.run([NVCC, *flags, "-c", str(WORK / src), "-o", str(obj)], check=True)
            objs2.append(str(obj))
        subprocess.run([NVCC, *flags, "-c", str(HERE / "ref_gpu_driver.cu"), "-o", str(drv)], check=True)
        subprocess.run([NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-o", str(OUT / f"kpz_ref_gpu_{tag}"),
                        str(drv), *objs2, *cpu, "-Xcompiler", "-pthread", "-lcudart"], check=True)
        print(f"built {OUT / f'kpz_ref_gpu_{tag}'}")
    param.write_text(t)


def build_adapter(cpu_objs: list[str], flags: list[str]) -> None:
    """tests/cpp/scheduler_b200_adapter.cpp -- a SchedulerService subclass forwarding to this
    library's C ABI -- against the reference's headers and CPU objects, into
    oracle/_ref/kpz_ref_adapter (needs cudakpz_b200/libkpzb200.so, built first)."""
    lib = HERE.parent / "cudakpz_b200" / "libkpzb200.so"
    if not lib.exists():
        print("libkpzb200.so not built; skipping the adapter", file=sys.stderr)
        return
    src = HERE.parent / "tests" / "cpp" / "scheduler_b200_adapter.cpp"
    obj = WORK / "scheduler_b200_adapter.o"
    subprocess.run(["g++", *flags, f"-I{HERE.parent / 'include'}", "-c", str(src), "-o", str(obj)], check=True)
    cpu = [o for o in cpu_objs if not o.endswith("ref_driver.o")]
    subprocess.run(["g++", "-pthread", "-o", str(OUT / "kpz_ref_adapter"), str(obj), *cpu,
                    f"-L{lib.parent}", "-lkpzb200", f"-Wl,-rpath,{lib.parent}"], check=True)
    print(f"built {OUT / 'kpz_ref_adapter'}")


def main() -> int:
    if not REF.is_dir():
        print(f"{REF} not present; skipping the reference build", file=sys.stderr)
        return 0
    if WORK.exists():
        shutil.rmtree(WORK)
    WORK.mkdir(parents=True)
    shutil.copytree(REF / "kpz", WORK / "kpz")
    shutil.copytree(REF / "inc", WORK / "inc")
    patch(WORK)
    OUT.mkdir(exist_ok=True)
    objs = []
    flags = ["-O2", "-std=c++14", "-w", "-DDSFMT_MEXP=19937", "-DKPZ_SWITCH_RNG=SLCG64",
             f"-I{WORK / 'kpz'}", f"-I{WORK / 'inc'}", "-include", str(WORK / "stub_io.h"), "-pthread"]
    for src in SOURCES:
        path = WORK / src
        obj = WORK / (path.stem + ".o")
        cc = ["gcc", "-O2", "-w", f"-I{WORK / 'inc'}"] if src.endswith(".c") else ["g++", *flags]
        extra = ["-Dprotected=public"] if ("schedulerCPUCB_instances" in src or "schedulerCPUDTr" in src) else []
        subprocess.run([*cc, *extra, "-c", str(path), "-o", str(obj)], check=True)
        objs.append(str(obj))
    drv = WORK / "ref_driver.o"
    subprocess.run(["g++", *flags, f"-I{HERE}", "-c", str(HERE / "ref_driver.cpp"), "-o", str(drv)], check=True)
    # the decision-injection unit (the reference's CBBit scheduler with a stand-in generator fed by
    # the oracle's restatement of the counter stream) and that restatement itself
    inj = WORK / "ref_inject.o"
    subprocess.run(["g++", *flags, "-Dprotected=public", f"-I{HERE}", "-c", str(HERE / "ref_inject.cpp"), "-o",
                    str(inj)], check=True)
    orc = WORK / "kpz_oracle.o"
    subprocess.run(["gcc", "-O2", "-std=c11", "-c", str(HERE / "kpz_oracle.c"), "-o", str(orc)], check=True)
    subprocess.run(["g++", "-pthread", "-o", str(OUT / "kpz_ref"), str(drv), str(inj), str(orc), *objs, "-lm"],
                   check=True)
    print(f"built {OUT / 'kpz_ref'}")
    build_adapter(objs, flags)
    build_gpu(objs)
    return 0


if __name__ == "__main__":
    sys.exit(main())
