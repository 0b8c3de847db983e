"""Test infrastructure only: build recipe for everything under oracle/.

* ``build_port()`` compiles the C restatement of the reference kernels
  (oracle/wadg_ref.c) into oracle/_build/libwadg_oracle.so.  It has no
  dependency on the reference tree and is rebuilt on any machine.

* ``build_ref()`` compiles the reference itself from its own sources (only
  where the reference checkout exists, i.e. not on a GPU host) into
  oracle/_ref/:
    - libwadgref_ops.so : operators.cpp + operators_c.cpp (Eigen 3.3.4 from
      the reference's vendor/ tarball, unpacked into oracle/_ref/) plus the
      ctypes wrapper oracle/ref_ops_api.cpp; oracle/ref_shim.h stands in for
      the MPI/Lua-dependent types.h.
    - libokl_<file>_N<N>.so : each OKL file rewritten by okl_to_cpp.py and
      compiled with g++ -O3 -fopenmp for one polynomial degree, with the
      kernel constants euler.c:2879-2950 would pass as OCCA defines.

Nothing here is run by the product; oracle/_ref/ stays out of git history
but ships with built artefacts so the CPU baseline can run next to the GPU.
"""

from __future__ import annotations

import ctypes
import os
import shutil
import subprocess
import sys
import tarfile

HERE = os.path.dirname(os.path.abspath(__file__))
# the reference checkout: $WADG_REFERENCE_DIR, else a directory named
# "reference" beside the repository's own (absent on GPU hosts)
REF_DIR = os.environ.get("WADG_REFERENCE_DIR",
                         os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference"))
OUT_REF = os.path.join(HERE, "_ref")
OUT_PORT = os.path.join(HERE, "_build")

DEGREES = {2: (1, 2, 3, 4), 3: (1, 2, 3, 4)}
OKL_FILES = {2: ("Euler2D.okl",), 3: ("Euler3D.okl", "Euler3Daffine.okl")}
GAMMA = "1.4"
TAU = "1.0"


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("command failed: " + " ".join(cmd) + "\n" + r.stdout + r.stderr)


def _stale(out, srcs):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(s) > t for s in srcs)


def build_port(verbose=False):
    os.makedirs(OUT_PORT, exist_ok=True)
    src = os.path.join(HERE, "wadg_ref.c")
    hdr = os.path.join(HERE, "wadg_ref.h")
    out = os.path.join(OUT_PORT, "libwadg_oracle.so")
    if _stale(out, [src, hdr, __file__]):
        _run(["gcc", "-O2", "-fPIC", "-shared", "-fopenmp", "-std=c11",
              "-ffp-contract=off", "-o", out, src, "-lm"])
        if verbose:
            print("built", out)
    return out


def reference_present():
    return os.path.isfile(os.path.join(REF_DIR, "operators.cpp"))


def _eigen_dir():
    tgz = os.path.join(REF_DIR, "vendor", "eigen-3.3.4.tar.gz")
    dst = os.path.join(OUT_REF, "eigen")
    if not os.path.isdir(dst):
        tmp = os.path.join(OUT_REF, "eigen_unpack")
        with tarfile.open(tgz) as tf:
            tf.extractall(tmp, filter="data")
        inner = [d for d in os.listdir(tmp) if d.startswith("eigen")][0]
        shutil.move(os.path.join(tmp, inner), dst)
        shutil.rmtree(tmp)
    return dst


def build_ref_ops(verbose=False):
    os.makedirs(OUT_REF, exist_ok=True)
    out = os.path.join(OUT_REF, "libwadgref_ops.so")
    srcs = [os.path.join(REF_DIR, "operators.cpp"), os.path.join(REF_DIR, "operators_c.cpp"),
            os.path.join(HERE, "ref_ops_api.cpp"), os.path.join(HERE, "ref_shim.h")]
    if _stale(out, srcs):
        eig = _eigen_dir()
        _run(["g++", "-O2", "-fPIC", "-shared", "-std=c++14", "-w",
              "-include", os.path.join(HERE, "ref_shim.h"),
              "-I", REF_DIR, "-I", eig, "-o", out] + srcs[:3])
        if verbose:
            print("built", out)
    return out


def refelem_sizes(dim, N, M=None):
    lib = ctypes.CDLL(os.path.join(OUT_REF, "libwadgref_ops.so"))
    sz = (ctypes.c_int * 5)()
    lib.wadgref_refelem_sizes(dim, N, M if M is not None else 2 * N, sz)
    return list(sz)


def okl_defines(dim, N, sizes, kblk=1):
    Np, Nq, Nfq, Nfaces, NfqNf = sizes
    Nfp = N + 1 if dim == 2 else (N + 1) * (N + 2) // 2
    T = max(Nq, NfqNf)
    log2Nq = 0
    while (1 << log2Nq) < Nq:
        log2Nq += 1
    r32 = lambda n: (1 + ((n - 1) >> 5)) * 32
    d = {
        "dfloat": "double", "USE_DOUBLE": "1", "p_DFLOAT_DOUBLE": "1",
        "uintloc_t": "unsigned int", "p_DFLOAT_MAX": "1.7976931348623157e308",
        "p_KblkU": kblk, "p_KblkV": kblk, "p_KblkS": kblk, "p_KblkF": kblk,
        "p_TAU": TAU, "p_T": T, "p_gamma": GAMMA, "p_Np": Np, "p_Nq": Nq,
        "p_log2Nq": log2Nq, "p_ceilNq2": 1 << log2Nq, "p_NfqNfaces": NfqNf,
        "p_NfpNfaces": Nfp * Nfaces, "p_Nvgeo": 4 if dim == 2 else 9,
        "p_Nfgeo": 3 if dim == 2 else 4, "p_Nfaces": Nfaces,
        "p_Nfields": 4 if dim == 2 else 5, "p_Nfq": Nfq, "p_Nfp": Nfp,
        "pT32": r32(T), "pNfaces32": r32(Nfaces), "pNq32": r32(Nq),
        "pNfqNfaces32": r32(NfqNf),
        "pSum32": r32(T) + r32(Nfaces) + r32(Nq) + r32(NfqNf),
        "E_test": 1, "p_RANK": 0,
    }
    return [f"-D{k}={v}" for k, v in d.items()]


def build_ref_okl(verbose=False):
    sys.path.insert(0, HERE)
    import okl_to_cpp  # noqa: E402

    built = []
    for dim, files in OKL_FILES.items():
        for fname in files:
            src = os.path.join(REF_DIR, "okl", fname)
            cpp = os.path.join(OUT_REF, fname.replace(".okl", ".cpp"))
            if _stale(cpp, [src, os.path.join(HERE, "okl_to_cpp.py")]):
                with open(src) as f:
                    text = f.read()
                with open(cpp, "w") as f:
                    f.write(okl_to_cpp.translate(text, fname))
            for N in DEGREES[dim]:
                out = os.path.join(OUT_REF, f"libokl_{fname[:-4]}_N{N}.so")
                if _stale(out, [cpp]):
                    sizes = refelem_sizes(dim, N)
                    _run(["g++", "-O3", "-fPIC", "-shared", "-fopenmp", "-w",
                          "-ffp-contract=off", "-o", out, cpp] + okl_defines(dim, N, sizes))
                    if verbose:
                        print("built", out)
                built.append(out)
    return built


def build_ref(verbose=False):
    if not reference_present():
        return False
    build_ref_ops(verbose)
    build_ref_okl(verbose)
    return True


if __name__ == "__main__":
    build_port(verbose=True)
    print("reference built:", build_ref(verbose=True))
