"""Test infrastructure only (oracle): rewrite the reference's OKL kernels into
plain C++ so that they compile with g++ straight from their own sources.

The OKL used by okl/Euler2D.okl, okl/Euler3D.okl and okl/Euler3Daffine.okl is
C plus five syntactic extensions, and these kernels use no `exclusive`
variables, so the rewrite is purely lexical and keeps every statement of the
reference in place:

  * ``kernel void f(...)``            -> ``extern "C" void f(...)``
  * ``for (a; b; c; outer0)``         -> ``#pragma omp parallel for`` + ``for (a; b; c)``
  * ``for (a; b; c; innerN)``         -> ``for (a; b; c)``   (sequential threads)
  * ``shared T x[..]``                -> ``T x[..]``  (local to the outer iteration)
  * ``barrier(localMemFence);``       -> ``;``  (inner-loop nests already run to
                                          completion one after the other)
  * ``restrict``                      -> ``__restrict__``
  * ``1.fe-4`` style literals          -> ``1e-4f`` (the float-suffixed constant
                                          the author wrote; the log-mean branch
                                          threshold, Euler3Daffine.okl:65)

This is the execution model of OCCA's Serial/OpenMP backends (outer loops
across cores, inner loops run in order inside one outer iteration), which is
how the reference runs on a CPU.

The minimal source patches needed for a correct FP64 reference are applied by
line number and checked against the expected original text, so a changed
reference fails loudly instead of being patched blindly:

  * okl/Euler3D.okl:57  ``#ifdef TESTING`` -> ``#if 0``   correct log-mean
  * okl/Euler2D.okl:38  ``#ifdef TESTING`` -> ``#if 0``   correct log-mean
  * okl/Euler2D.okl:106 ``#ifdef TESTING`` -> ``#if 0``   real two-point flux
    (under TESTING euler2d_flux returns the constants 1..4, Euler2D.okl:106-138)

The rest of both files keeps its shipped TESTING configuration (its loop code
is the variant that compiles).

Only the kernels on the hot path (and Euler3D.okl's per-element kinetic-energy
diagnostic, euler_3d_compute_aux) are kept (``KERNELS``): everything before the
first ``kernel`` (macros, logmean, VU/UV, the flux functions) plus each listed
kernel from its ``kernel void`` line up to the next one.  Other kernels of
Euler3D.okl are experiments that do not all compile (e.g. its own
euler_update_3d reads an undeclared ``max_iter`` under TESTING, :3524).
"""

from __future__ import annotations

import re
import sys

PATCHES = {
    "Euler3D.okl": [(57, "#ifdef TESTING", "#if 0")],
    "Euler2D.okl": [(38, "#ifdef TESTING", "#if 0"), (106, "#ifdef TESTING", "#if 0")],
    "Euler3Daffine.okl": [],
}

KERNELS = {
    "Euler3Daffine.okl": ("euler_vol_3d", "euler_surf_3d", "euler_update_3d"),
    "Euler3D.okl": ("euler_vol_3d_curved", "euler_surf_3d", "euler_update_3d_curved",
                    "euler_3d_compute_aux"),
    "Euler2D.okl": ("euler_vol_2d", "euler_vol_2d_curved", "euler_surf_2d",
                    "euler_update_2d", "euler_update_2d_curved"),
}

PRELUDE = r"""// generated from a reference OKL file by oracle/okl_to_cpp.py; do not edit
#include <cmath>
#include <cstdio>
using std::sqrt; using std::log; using std::exp; using std::pow; using std::fabs;
static inline double max(double a, double b) { return a > b ? a : b; }
static inline double min(double a, double b) { return a < b ? a : b; }
#define atomicAdd(ptr, val) (*(ptr) += (val))
"""

_FOR = re.compile(r"for\s*\(([^;{}]*);([^;{}]*);([^;{}]*);\s*(outer|inner)(\d+)\s*\)")


def _for(m: re.Match) -> str:
    head = f"for ({m.group(1).strip()}; {m.group(2).strip()}; {m.group(3).strip()})"
    if m.group(4) == "outer":
        return "\n#pragma omp parallel for schedule(static)\n" + head
    return head


def _select(src: str, keep) -> str:
    if keep is None:
        return src
    starts = [m.start() for m in re.finditer(r"^kernel\s+void\s", src, re.M)]
    if not starts:
        return src
    parts = [src[: starts[0]]]
    found = set()
    for a, b in zip(starts, starts[1:] + [len(src)]):
        m = re.match(r"kernel\s+void\s+(\w+)", src[a:b])
        if m and m.group(1) in keep:
            parts.append(src[a:b])
            found.add(m.group(1))
    missing = set(keep) - found
    if missing:
        raise SystemExit(f"kernels not found: {sorted(missing)}")
    return "".join(parts)


def translate(text: str, name: str) -> str:
    lines = text.split("\n")
    for lineno, old, new in PATCHES.get(name, []):
        got = lines[lineno - 1].strip()
        if got != old:
            raise SystemExit(f"{name}:{lineno}: expected {old!r}, found {got!r}")
        lines[lineno - 1] = lines[lineno - 1].replace(old, new)
    src = _select("\n".join(lines), KERNELS.get(name))
    src = re.sub(r"\bkernel\s+void\b", 'extern "C" void', src)
    src = _FOR.sub(_for, src)
    src = re.sub(r"\bshared\s+(?=(dfloat|int|double|float)\b)", "", src)
    src = re.sub(r"\bbarrier\s*\(\s*(local|global)MemFence\s*\)\s*;", ";", src)
    src = re.sub(r"\brestrict\b", "__restrict__", src)
    src = re.sub(r"\b(\d+)\.fe-(\d+)", r"\1e-\2f", src)
    return PRELUDE + src


def main(argv):
    inp, out = argv[1], argv[2]
    name = inp.rsplit("/", 1)[-1]
    with open(inp) as f:
        text = f.read()
    with open(out, "w") as f:
        f.write(translate(text, name))


if __name__ == "__main__":
    main(sys.argv)
