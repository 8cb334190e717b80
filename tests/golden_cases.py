"""Load the QL golden fixtures written by tests/golden/make_golden.py (the DNS
fixtures, dns_*.npz from make_dns_golden.py, are read by the DNS tests)."""
import glob
import os

import numpy as np

from ql_dns_b200.params import QLParams

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def names():
    return sorted(os.path.basename(f)[:-4] for f in glob.glob(os.path.join(GOLDEN, "*.npz"))
                  if not os.path.basename(f).startswith("dns_"))


def load(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    p = QLParams(model=int(z["model"]), integrator=int(z["integrator"]), nx=int(z["nx"]), ny=int(z["ny"]),
                 NZ=int(z["NZ"]), L=tuple(float(v) for v in z["L"]), q=float(z["q"]), omega=float(z["omega"]),
                 nu=float(z["nu"]), eta=float(z["eta"]), B0z=float(z["B0z"]),
                 viscosity_order=int(z["viscosity_order"]), dt=float(z["dt"]), remap=int(z["remap"]),
                 quasilinear=int(z["quasilinear"]))
    return p, {k: z[k] for k in z.files}
