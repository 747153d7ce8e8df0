"""Pivot-step phase clocks of the blocked RRQR (k_rrqr_blk) on the bench
workload: runs factorizations through libspaqr_b200_rrqrclk.so (the library
built with -DSPQ_RRQR_CLOCKS: `make -C spaqr_public_b200/csrc rrqrclk`) and
prints, per precision, the clock64() cycles of each phase of one pivot step of
one CTA, averaged over all CTA-steps of a warmed factorization.

    python spaqr_public_b200/csrc/bench/rrqr_phases.py [workload]
"""
import ctypes as C
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", "..", ".."))
sys.path.insert(0, ROOT)

import spaqr_public_b200._abi as abi  # noqa: E402

abi.LIB_PATH = os.path.join(ROOT, "spaqr_public_b200", "_build", "libspaqr_b200_rrqrclk.so")

from spaqr_public_b200 import FP32, FP64, Tree, matgen  # noqa: E402

PHASES = ["arg-max over the slab", "cluster barrier wait", "candidate reduction + F(:, pc)",
          "pivot column + reflector", "partial products C_bs^T x", "row update + norm downdates",
          "norm recomputation"]


def main():
    name = sys.argv[1] if len(sys.argv) > 1 else "advdiff3d_64"
    w = matgen.workload(name)
    A = matgen.column_normalize(w["A"])
    L = abi.lib()
    L.spq_rrqr_phase_clocks.restype = C.c_int
    L.spq_rrqr_phase_clocks.argtypes = [C.POINTER(C.c_ulonglong), C.c_int]
    buf = (C.c_ulonglong * 16)()
    for prec, label in ((FP32, "FP32"), (FP64, "FP64")):
        for it in range(5):  # the autotuner settles in the first factorizations
            t = Tree(w["levels"], w["skip"], precision=prec)
            t.set_tol(w["tol"])
            t.set_scale(1)
            t.set_square(1)
            t.set_coords_grid(w["n"], w["d"])
            t.partition(A)
            t.assemble(A)
            if L.spq_rrqr_phase_clocks(buf, 1):
                raise RuntimeError("reading the phase clocks failed")
            t.factorize()
            if L.spq_rrqr_phase_clocks(buf, 0):
                raise RuntimeError("reading the phase clocks failed")
            t.close()
        v = [float(x) for x in buf]
        steps, blocks = max(v[8], 1.0), max(v[9], 1.0)
        tot = sum(v[:8])
        print(f"{label} {name}: {int(v[8])} CTA-steps, {int(v[9])} CTA-blocks, "
              f"{sum(v[:7]) / steps:.0f} cycles per CTA-step + {v[7] / blocks:.0f} per block end")
        for i, ph in enumerate(PHASES):
            print(f"  {ph:32s} {v[i] / steps:8.0f} cycles/step  {100 * v[i] / tot:5.1f} %")
        print(f"  {'block end (C -= V_b F^T)':32s} {v[7] / steps:8.0f} cycles/step  {100 * v[7] / tot:5.1f} %")


if __name__ == "__main__":
    main()
