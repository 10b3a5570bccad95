"""Oracle collision matrices of the production-size workloads, as committed fixtures.

    OPENBLAS_NUM_THREADS=<cores> python tests/golden/make_production_u.py [--sweep] [nch ...]

For each channel count (default: 128, i.e. N = 25600) this runs the FP64 oracle (LAPACK
zgesv through scipy, the reference's Type 1 path) on the seeded production workload of
``hprmat_b200.workloads`` and writes ``production_u_nch<nch>.npz`` next to this script:
the collision matrix U (nopen x nopen), nopen, the seed, and the oracle's own relative
residual ||B - C X||_F / ||B||_F.  With ``--sweep`` the workload is the precision sweep's
generator (closed-channel thresholds at 40 MeV, ``workloads.sweep``) and the files are
``sweep_u_nch<nch>.npz``.  The N = 25600 solve takes a few minutes on 8 cores.
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from hprmat_b200 import workloads  # noqa: E402
from oracle import rmatrix_oracle as orc  # noqa: E402


def main(nchs, sweep=False):
    for nch in nchs:
        w = workloads.sweep(nch) if sweep else workloads.production(nch=nch)
        t = time.time()
        mesh = orc.rmat_ini(w.nr, 1, w.rmax)
        res = orc.rmatrix(w.nch, w.lval, w.qk, w.eta, w.rmax, mesh, w.cpot)
        bnd = res.boundary
        C = orc.assemble(mesh, 1, w.nch, w.lval, w.qk, bnd.xc, w.cpot)
        B = orc.surface_rhs(mesh.q2[:, 0].astype(np.complex128), w.nch)
        relres = np.linalg.norm(B - C @ res.x) / np.linalg.norm(B)
        dt = time.time() - t
        out = os.path.join(HERE, f"{'sweep' if sweep else 'production'}_u_nch{nch}.npz")
        np.savez_compressed(out, u=res.cu, nopen=res.nopen, seed=2 if sweep else 1, nch=nch, relres=relres,
                            seconds=dt)
        print(f"nch={nch} N={w.n} nopen={res.nopen} relres={relres:.3e} {dt:.1f}s -> {out}")


if __name__ == "__main__":
    args = [a for a in sys.argv[1:] if a != "--sweep"]
    main([int(a) for a in args] or [128], sweep="--sweep" in sys.argv[1:])
