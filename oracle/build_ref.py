"""Build recipe for oracle/_ref: the reference's own HighOrder code on CPU.

TEST INFRASTRUCTURE ONLY.  For each CPU grid tag this script makes a folder
oracle/_ref/<tag>/ holding symlinks to the reference sources where they lie
(TD_GPU_code/HighOrder/{kern.cu,mycmplx.h,main.c,proj.c}) and a grid header
parm.h with the tag's N, M, Xmin, Xmax (the reference fixes these at compile
time in HighOrder/parm.h:1-13; the "ho" tag links the reference's own
parm.h unchanged).  It then compiles them with oracle/ref_emu/ into
oracle/_ref/libref_<tag>.so.  For each GPU tag it links body.cu and kern.cu
as well, compiled unchanged by nvcc for sm_100a, with the driver
oracle/ref_gpu/ref_gpu_main.cpp into the executable oracle/_ref/refgpu_<tag>
(the reference's own GPU code, run on the B200 as the reference-GPU
baseline and for the host-loop fixture).  Nothing is copied out of the
reference tree and nothing is written outside oracle/_ref/.  The "dropin"
tag links the reference's main.c and proj.c with this repository's
bh_ringdown_b200/integration/body_bhr.c against libbhr.so into
oracle/_ref/dropin_run (the drop-in as a maintainer would build it).  The
"genot" tag compiles the reference's trajectory generator, GenOT/
ParamWLMino.cc and GenOT/WL_BL.cc, where they lie, as GenOT/README:30-31
does (g++ ... -lm), into oracle/_ref/genot/{ParamWLMino,WL_BL}.

Usage: python oracle/build_ref.py [--ref <reference root>] [tag ...]

The reference root is --ref, else $BHR_REFERENCE_ROOT, else a directory
named `reference` beside this repository's root.
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
EMU = os.path.join(HERE, "ref_emu")

# Grid tags: (N, M, Xmin, Xmax) or None for the reference's own parm.h.
TAGS = {
    "ho": None,                           # 16000 x 256 on [-50, 50]
    "pin": (256, 32, -50.0, 50.0),        # small reference-domain pin grid
    "c1s": (512, 64, -100.0, 300.0),      # config-1 domain, reduced grid
    "cfg2": (8192, 128, -200.0, 600.0),   # plunge-ringdown workload grid
    "p16k": (16384, 256, -200.0, 600.0),  # the same domain at 16384 x 256 (the default bench workload)
}
DEFAULT_TAGS = ("pin", "c1s", "cfg2", "p16k", "gpin", "gp16k", "dropin", "genot")

# main.c defines globals with the same names as kern.cu's device scalars;
# they are renamed at compile time so both link into one library.
MAIN_RENAMES = ["mass", "aa", "ss", "mm", "dx", "dtheta", "timer", "dt", "delta"]


def grid_header(n: int, m: int, xmin: float, xmax: float) -> str:
    return (
        f"#define N {n}\n#define M {m}\n#define Xmax {xmax!r}\n#define Xmin {xmin!r}\n"
        "#define Text 90.0\n#define Nd 100\n#define Fr 50\n#define T  1500.0\n"
        "#define PTSX 128\n#define PTSY 128\n#define Pi 3.14159265358979\n"
        "#define idx(b,a) (N*(b)+(a))\n"
    )


def run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")


def build_tag(ref_root: str, tag: str) -> str:
    ho = os.path.join(ref_root, "TD_GPU_code", "HighOrder")
    d = os.path.join(OUT, tag)
    os.makedirs(d, exist_ok=True)
    names = ["kern.cu", "mycmplx.h", "main.c", "proj.c"] + (["parm.h"] if TAGS[tag] is None else [])
    for name in names:
        link = os.path.join(d, name)
        if os.path.lexists(link):
            os.remove(link)
        os.symlink(os.path.join(ho, name), link)
    if TAGS[tag] is not None:
        with open(os.path.join(d, "parm.h"), "w") as f:
            f.write(grid_header(*TAGS[tag]))
    lib = os.path.join(OUT, f"libref_{tag}.so")
    drv_o, main_o, proj_o = (os.path.join(d, x) for x in ("driver.o", "main.o", "proj.o"))
    run(["g++", "-O2", "-fopenmp", "-fPIC", "-w", "-std=c++17", "-include", os.path.join(EMU, "prelude.h"),
         "-I", d, "-c", os.path.join(EMU, "ref_driver.cpp"), "-o", drv_o])
    defs = [f"-D{v}=hmc_{v}" for v in MAIN_RENAMES] + ["-Dmain=hmc_main", "-Dbody=hmc_body"]
    run(["gcc", "-O2", "-fPIC", "-w", *defs, "-c", os.path.join(d, "main.c"), "-o", main_o])
    run(["gcc", "-O2", "-fPIC", "-w", "-c", os.path.join(d, "proj.c"), "-o", proj_o])
    run(["g++", "-shared", "-fopenmp", "-o", lib, drv_o, main_o, proj_o, "-lm"])
    return lib


def default_reference_root() -> str:
    """$BHR_REFERENCE_ROOT, else `reference` beside the repository root."""
    return os.environ.get("BHR_REFERENCE_ROOT",
                          os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference"))


# GPU builds of the reference itself (body.cu + kern.cu compiled unchanged by
# nvcc for sm_100a, with oracle/ref_gpu/ref_gpu_main.cpp in place of main()'s m
# loop): (N, M, Xmin, Xmax, T, Fr).  T fixes the step count, as parm.h does.
GPU_TAGS = {
    "gpin": (256, 32, -50.0, 50.0, 300.0, 50),         # host-loop fixture: rows from k dt >= Xmax + 200
    "gp16k": (16384, 256, -200.0, 600.0, 4.4, 50),     # the default bench grid, ~1000 steps
}
NVCC_ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def gpu_grid_header(n, m, xmin, xmax, t, fr):
    return grid_header(n, m, xmin, xmax).replace("#define Fr 50\n#define T  1500.0\n",
                                                 f"#define Fr {fr}\n#define T  {t!r}\n")


def build_gpu_tag(ref_root: str, tag: str) -> str:
    ho = os.path.join(ref_root, "TD_GPU_code", "HighOrder")
    d = os.path.join(OUT, tag)
    os.makedirs(d, exist_ok=True)
    for name in ["kern.cu", "body.cu", "mycmplx.h", "main.c", "proj.c"]:
        link = os.path.join(d, name)
        if os.path.lexists(link):
            os.remove(link)
        os.symlink(os.path.join(ho, name), link)
    with open(os.path.join(d, "parm.h"), "w") as f:
        f.write(gpu_grid_header(*GPU_TAGS[tag]))
    exe = os.path.join(OUT, f"refgpu_{tag}")
    o = {k: os.path.join(d, k + ".o") for k in ("kern", "body", "main", "proj", "drv")}
    nv = ["nvcc", *NVCC_ARCH, "-O3", "-w", "-I", d]
    # body.cu writes two bytes into its one-byte `snum` (HighOrder/body.cu:61,67);
    # without fortified sprintf that stays the reference's own behaviour instead of an abort
    run(nv + ["-c", os.path.join(d, "kern.cu"), "-o", o["kern"]])
    run(nv + ["-Xcompiler", "-U_FORTIFY_SOURCE", "-c", os.path.join(d, "body.cu"), "-o", o["body"]])
    # main.c and proj.c as HighOrder/build.sh compiles them (g++, C++ linkage)
    defs = [f"-D{v}=hmc_{v}" for v in MAIN_RENAMES] + ["-Dmain=hmc_main"]
    run(["g++", "-x", "c++", "-O2", "-w", *defs, "-I", d, "-c", os.path.join(d, "main.c"), "-o", o["main"]])
    run(["g++", "-x", "c++", "-O2", "-w", "-c", os.path.join(d, "proj.c"), "-o", o["proj"]])
    run(["g++", "-O2", "-std=c++17", "-Wall", "-I", d, "-c", os.path.join(HERE, "ref_gpu", "ref_gpu_main.cpp"),
         "-o", o["drv"]])
    run(["nvcc", *NVCC_ARCH, "-o", exe, o["drv"], o["body"], o["kern"], o["main"], o["proj"], "-lm"])
    return exe


# The drop-in: the reference's own main.c (its m = -5..5 loop, aa = 1e-8,
# dt = 0.002, HighOrder/main.c:40-55) and proj.c, with
# bh_ringdown_b200/integration/body_bhr.c in place of body.cu and kern.cu,
# linked to libbhr.so, for a small grid: (N, M, Xmin, Xmax, T, Fr).
DROPIN_TAGS = {"dropin": (256, 32, -50.0, 50.0, 270.0, 50)}


def build_dropin_tag(ref_root: str, tag: str) -> str:
    ho = os.path.join(ref_root, "TD_GPU_code", "HighOrder")
    d = os.path.join(OUT, tag)
    os.makedirs(d, exist_ok=True)
    for name in ["main.c", "proj.c"]:
        link = os.path.join(d, name)
        if os.path.lexists(link):
            os.remove(link)
        os.symlink(os.path.join(ho, name), link)
    with open(os.path.join(d, "parm.h"), "w") as f:
        f.write(gpu_grid_header(*DROPIN_TAGS[tag]))
    repo = os.path.dirname(HERE)
    libdir = os.path.join(repo, "bh_ringdown_b200")
    if not os.path.exists(os.path.join(libdir, "libbhr.so")):
        raise RuntimeError("build libbhr.so first (make -C bh_ringdown_b200/csrc)")
    exe = os.path.join(OUT, f"{tag}_run")
    objs = []
    # as HighOrder/build.sh: g++ -O -c main.c proj.c (C++ linkage), then body_bhr.c the same way
    for src in (os.path.join(d, "main.c"), os.path.join(d, "proj.c"),
                os.path.join(repo, "bh_ringdown_b200", "integration", "body_bhr.c")):
        obj = os.path.join(d, os.path.basename(src).replace(".c", ".o"))
        run(["g++", "-x", "c++", "-O", "-w", "-I", d, "-I", os.path.join(repo, "include"), "-c", src, "-o", obj])
        objs.append(obj)
    rpath = os.path.relpath(libdir, OUT)
    run(["g++", "-o", exe, *objs, "-L" + libdir, "-lbhr", f"-Wl,-rpath,$ORIGIN/{rpath}", "-lm"])
    return exe


# The reference's trajectory generator, its two programs built as its README
# says (GenOT/README:30-31).
GENOT_PROGRAMS = ("ParamWLMino", "WL_BL")


def build_genot(ref_root: str, tag: str = "genot") -> str:
    d = os.path.join(OUT, tag)
    os.makedirs(d, exist_ok=True)
    for prog in GENOT_PROGRAMS:
        run(["g++", "-O2", "-w", os.path.join(ref_root, "GenOT", prog + ".cc"), "-o", os.path.join(d, prog), "-lm"])
    return d


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=default_reference_root())
    ap.add_argument("tags", nargs="*", default=list(DEFAULT_TAGS))
    args = ap.parse_args(argv)
    if not os.path.isdir(os.path.join(args.ref, "TD_GPU_code", "HighOrder")):
        print(f"build_ref: reference not found at {args.ref}; skipping", file=sys.stderr)
        return 0
    known = sorted(TAGS) + sorted(GPU_TAGS) + sorted(DROPIN_TAGS) + ["genot"]
    bad = [t for t in args.tags if t not in known]
    if bad:
        print(f"unknown tags {bad}; known {known}", file=sys.stderr)
        return 2
    os.makedirs(OUT, exist_ok=True)

    def build(t):
        if t in TAGS:
            return build_tag(args.ref, t)
        if t == "genot":
            return build_genot(args.ref, t)
        return build_gpu_tag(args.ref, t) if t in GPU_TAGS else build_dropin_tag(args.ref, t)
    with ThreadPoolExecutor(max_workers=len(args.tags)) as ex:
        for lib in ex.map(build, args.tags):
            print("built", os.path.relpath(lib, os.path.dirname(HERE)))
    return 0


if __name__ == "__main__":
    sys.exit(main())
