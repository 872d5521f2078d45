"""Build the xns_b200 CUDA library (sm_100a) in-tree.

    python softx-d-16-00083_b200/build.py            # lib/libxns_b200.so
    python softx-d-16-00083_b200/build.py --shim     # + the drop-in calc-function shim and the
                                                     #   relinked XaNSoNS program (needs the
                                                     #   reference sources, REF=/path)

Every object is compiled for sm_100a only; nothing is JIT-compiled at run time.  Objects are rebuilt
only when a source or header is newer than the library.
"""
import argparse
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "lib")
BUILD = os.path.join(PKG, "_build")
INCLUDE = os.path.join(ROOT, "include")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
GENCODE = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = GENCODE + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I" + INCLUDE, "-I" + CSRC,
                        "-Xptxas", "-warn-spills"]

HOST_SOURCES = ["writers.cpp"]  # host-only parts of the library, in host/
SOURCES = ["context.cu", "schedule.cu", "hist.cu", "sinc_engine.cu", "debye.cu", "debye_tc.cu", "hist_iq.cu", "hist_split.cu", "pdf.cu",
           "amp2d.cu", "noalloc.cu", "tc_gemm.cu", "tc_exact.cu", "batch.cu", "mlp.cu", "learned.cu", "builder.cu",
           "rearrange.cu"]


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd):
    print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)


def build_lib(verbose_ptxas=False):
    os.makedirs(LIB, exist_ok=True)
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cuh")]
    headers.append(os.path.join(INCLUDE, "xns_b200.h"))
    objs = []
    for src in SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src.replace(".cu", ".o"))
        if _newer(o, [s] + headers):
            flags = NVCC_FLAGS + (["-Xptxas", "-v"] if verbose_ptxas else [])
            _run([NVCC] + flags + ["-c", s, "-o", o])
        objs.append(o)
    for src in HOST_SOURCES:
        s = os.path.join(PKG, "host", src)
        o = os.path.join(BUILD, src.replace(".cpp", ".o"))
        if _newer(o, [s, os.path.join(INCLUDE, "xns_b200.h")]):
            _run(["g++", "-O2", "-std=c++17", "-fPIC", "-Wall", "-I" + INCLUDE, "-c", s, "-o", o])
        objs.append(o)
    so = os.path.join(LIB, "libxns_b200.so")
    if _newer(so, objs):
        _run([NVCC] + GENCODE + ["-shared", "-o", so] + objs + ["-lcudart"])
    return so


# reference functions the relinked program takes from host/interpose.cpp (demangled name prefixes)
INTERPOSED = ("block::calcAtoms(", "RearrangementInt(", "printI(", "printPartialI(", "printI2(", "printPDF(",
              "printPartialPDF(", "printAtoms(")


def _weaken(obj, out, prefixes):
    """A copy of obj (built here from the reference's sources) in which the global functions whose
    demangled names start with prefixes are weak, so that a strong definition linked beside it wins."""
    lines = subprocess.check_output(["nm", "--defined-only", obj], text=True).splitlines()
    mangled = [l.split()[-1] for l in lines if len(l.split()) == 3 and l.split()[1] == "T"]
    demangled = subprocess.check_output(["c++filt"], input="\n".join(mangled), text=True).splitlines()
    weak = [m for m, d in zip(mangled, demangled) if d.startswith(prefixes)]
    _run(["objcopy"] + ["--weaken-symbol=" + m for m in weak] + [obj, out])


def build_shim(ref):
    """The drop-in: calc_functions_b200.cpp exports the reference's four CPU calc-function
    signatures (main.cpp:344-347) on top of libxns_b200.so.  It is compiled against the reference's
    own typedefs.h where it lies; the reference program is relinked from its own sources with
    CalcFunctions.cpp built -D UseCUDA (which drops exactly its CPU calc functions,
    CalcFunctions.cpp:546-1092) and main.cpp built without backend macros (so it calls those four)."""
    if not os.path.exists(os.path.join(ref, "typedefs.h")):
        print("reference sources not found at %s: shim not built" % ref)
        return None
    so = build_lib()
    shim_src = os.path.join(PKG, "host", "calc_functions_b200.cpp")
    shim_o = os.path.join(BUILD, "calc_functions_b200.o")
    cxx = "g++"
    if _newer(shim_o, [shim_src, os.path.join(INCLUDE, "xns_b200.h")]):
        _run([cxx, "-O2", "-std=c++11", "-fPIC", "-I" + ref, "-I" + INCLUDE, "-c", shim_src, "-o", shim_o])
    shim_so = os.path.join(LIB, "libxns_calc_shim.so")
    if _newer(shim_so, [shim_o, so]):
        _run([cxx, "-shared", "-o", shim_so, shim_o, "-L" + LIB, "-lxns_b200", "-Wl,-rpath,$ORIGIN"])
    objs = []
    for f, defs in (("main", []), ("tinyxml2", []), ("ReadXML", []), ("IO", []), ("CalcFunctions", ["-D", "UseCUDA"])):
        o = os.path.join(BUILD, "ref_" + f + ".o")
        s = os.path.join(ref, f + ".cpp")
        if _newer(o, [s]):
            _run([cxx, "-O3", "-std=c++11", "-w"] + defs + ["-I" + ref, "-c", s, "-o", o])
        objs.append(o)
    # the functions either side of the calc functions (builder, rearrangement correction, writers) are
    # not behind a macro: weaken them in copies of the reference's objects and link host/interpose.cpp's
    # definitions in their place
    ip_src = os.path.join(PKG, "host", "interpose.cpp")
    ip_o = os.path.join(BUILD, "interpose.o")
    if _newer(ip_o, [ip_src, os.path.join(INCLUDE, "xns_b200.h")]):
        _run([cxx, "-O2", "-std=c++11", "-I" + ref, "-I" + INCLUDE, "-c", ip_src, "-o", ip_o])
    linked = []
    for o in objs:
        if o.endswith("ref_CalcFunctions.o") or o.endswith("ref_IO.o"):
            w = o.replace(".o", "_weak.o")
            if _newer(w, [o]):
                _weaken(o, w, INTERPOSED)
            linked.append(w)
        else:
            linked.append(o)
    exe = os.path.join(LIB, "XaNSoNS_B200")
    if _newer(exe, linked + [ip_o, shim_so]):
        _run([cxx, "-o", exe] + linked + [ip_o, "-L" + LIB, "-lxns_calc_shim", "-lxns_b200", "-Wl,-rpath,$ORIGIN"])
    # test program for the drop-in structure builder (tests/shim/build_atoms_check.cpp)
    chk_src = os.path.join(ROOT, "tests", "shim", "build_atoms_check.cpp")
    chk = os.path.join(LIB, "xns_build_atoms_check")
    ref_cf = [o for o in objs if o.endswith("ref_CalcFunctions.o") or o.endswith("ref_IO.o")]
    if os.path.exists(chk_src) and _newer(chk, [chk_src, shim_so] + ref_cf):
        _run([cxx, "-O2", "-std=c++11", "-w", "-I" + ref, chk_src] + ref_cf +
             ["-o", chk, "-L" + LIB, "-lxns_calc_shim", "-lxns_b200", "-Wl,-rpath,$ORIGIN"])
    return exe


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--shim", action="store_true")
    ap.add_argument("--ref", default=os.environ.get("REF", ""),
                    help="the reference source tree (default: $REF); --shim needs it")
    ap.add_argument("--ptxas-v", action="store_true")
    a = ap.parse_args()
    print(build_lib(a.ptxas_v))
    if a.shim:
        if not a.ref:
            print("--shim: no reference source tree given (--ref or REF): shim not built")
        else:
            print(build_shim(a.ref))


if __name__ == "__main__":
    sys.exit(main())
