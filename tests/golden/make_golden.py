"""Generate tests/golden/transport_nxp3.npz.

No golden vectors exist in the reference for this path and its Fortran cannot
be compiled here, so these fixtures come from the independent numpy
restatement (tests/numpy_ref.py) on a tiny grid.  They pin the C++ oracle
and the GPU path to that restatement; regenerate only when the restatement
itself is corrected:  python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
sys.path.insert(0, os.path.dirname(HERE))

from olam_b200.synth.grid import build_grid, stretched_levels  # noqa: E402
from olam_b200.synth.state import transport_state  # noqa: E402
from numpy_ref import transport_plain  # noqa: E402

nxp, seed, dtlm = 3, 5, 1800.0
zz = stretched_levels(8, 100.0, 30000.0)
g = build_grid(nxp, zz, seed=seed)
st = transport_state(g, dtlm, 3, seed=seed)
out2 = transport_plain(g, st, st.tracers, st.sct, dtlm, nrk=2, order=2)
out3 = transport_plain(g, st, st.tracers, st.sct, dtlm, nrk=3, order=2)
np.savez_compressed(os.path.join(HERE, "transport_nxp3.npz"), nxp=nxp, seed=seed, dtlm=dtlm, zz=zz,
                    vmasc=st.vmasc, wmasc=st.wmasc, rho_old=st.rho_old, rho=st.rho, wc=st.wc,
                    tracers=st.tracers, sct=st.sct, out_rk2=out2, out_rk3=out3)
print("wrote", os.path.join(HERE, "transport_nxp3.npz"))
