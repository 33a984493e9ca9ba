"""Generates tests/golden/adjoint_tlm.npz: the tangent-linear reference
gradient of the adjoint workload (tests/_util.py ADJOINT_*).

The reference solver compiled with a dual-number scalar (oracle/ref_tlm.cpp,
oracle/_ref/libdgsem_ref_tlm.so) runs its own SSPRK3 for ADJOINT_STEPS steps
from the seeded initial state, once per seeded momentum direction d_k, and
returns J = mean kinetic energy of the final state and the exact directional
derivative dJ/du0 . d_k.  The fixture stores J and the 8 derivatives.
Regenerate with:  make -C oracle ref && python tests/golden/make_adjoint_golden.py
"""
from __future__ import annotations

import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import ref_tlm_binding as tb  # noqa: E402
from tests import _util as U  # noqa: E402


def main() -> None:
    s, u0 = U.adjoint_initial_state()
    c = U.ADJOINT_CASE
    tc = tb.TangentCase(tb.NS2D, c["polydeg"], c["cells"], c["left"], c["right"], 1.4, c["mu"],
                        c["prandtl"])
    dirs = U.adjoint_directions(u0)
    J = None
    dJ = []
    for k, d in enumerate(dirs):
        t0 = time.time()
        Jk, dk = tc.objective(u0, d, 0.0, U.ADJOINT_DT, U.ADJOINT_STEPS)
        J = Jk if J is None else J
        assert Jk == J
        dJ.append(dk)
        print(f"direction {k}: dJ = {dk:.17e} ({time.time() - t0:.1f} s)")
    np.savez(os.path.join(HERE, "adjoint_tlm.npz"), J=np.float64(J), dJ=np.array(dJ),
             steps=U.ADJOINT_STEPS, dt=U.ADJOINT_DT)
    print("J =", repr(J))


if __name__ == "__main__":
    main()
