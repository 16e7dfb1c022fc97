"""Load a golden fixture (tests/golden/*.npz) into the objects the reference API takes."""

import os

import numpy as np

from exmarg_b200 import synth

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


class Fixture:
    def __init__(self, name):
        z = np.load(os.path.join(GOLDEN, name + ".npz"))
        self.z = z
        self.name = name
        self.seg = dict(d_H=z["d_H"], d_L=z["d_L"], f=z["f"], nu=z["nu"], sig2=z["sig2"], T=float(z["T"]),
                        fmin=float(z["fmin"]), fmax=float(z["fmax"]))
        self.rows = z["bank_rows"]
        self.W, self.u = z["W"], z["u"]
        self.lo, self.n_time = int(z["lo"]), int(z["n_time"])
        self.spec = synth.TableSpec(ntau=int(z["ntau"]), nphif=49, nb=int(z["nb"]), nd=int(z["nd"]))
        self.s_nodes = z["s_nodes"]
        fac = (z["fac_M"], z["fac_P"], z["fac_Q"], z["fac_S"])
        tables = [synth.gen_table_node(self.spec, k, self.s_nodes, int(z["tab_seed"]), fac)
                  for k in range(self.s_nodes.size)]
        self.store = synth.MemoryStore(self.spec, self.s_nodes, int(z["tab_seed"]), tables=tables)
        self.ymin = float(z["ymin"])
        self.prior = str(z["prior"])
        self.density = (z["dens_lny"], z["dens_p"]) if "dens_lny" in z else None
        self.n_loud, self.n_random = int(z["n_loud"]), int(z["n_random"])
        self.ln_lambda, self.ln_b = z["ln_lambda"], z["ln_b"]

    @property
    def prior_arg(self):
        return self.density if self.density is not None else self.prior

    def b200_bank(self):
        from exmarg_b200 import MassBank
        M, q, chi = (self.rows[:, i] for i in range(3))
        return MassBank(M, q, chi, self.seg, "b200", W=self.W, u=self.u)
