"""Shared helpers of the parity tests: run the oracle and the engine on the
same inputs and measure the per-field error the way the acceptance bar is
stated (relative L2 over all stored complex entries)."""
import os

import numpy as np

import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")


def rel_l2(a, b) -> float:
    a = np.asarray(a)
    b = np.asarray(b)
    nb = np.linalg.norm(b)
    if nb == 0.0:
        return float(np.linalg.norm(a))
    return float(np.linalg.norm(a - b) / nb)


def oracle_cfg(desc, threaded=False) -> "O.Config":
    return O.Config(Nx=desc.Nx, Nz=desc.Nz, ny=desc.ny, Re=desc.Re, alp=desc.alp, bet=desc.bet,
                    mpgx=desc.mpgx, flag_ctpress=desc.flag_ctpress, grid_type=desc.grid_type,
                    dyq=desc.dyq, ppp=desc.ppp, gamma=desc.gamma, dt_mode=desc.dt_mode, CFL=desc.CFL,
                    dt_fixed=desc.dt)


def golden_ic():
    z = np.load(os.path.join(GOLDEN, "ref_ic_0032x0032x0153.npz"))
    return z["u1"], z["u2"], z["u3"], z["p"]


# Per-field errors of every parity case of a run, in the order the cases ran;
# written out by the session hook in conftest.py when LH_PARITY_OUT names a
# file (a JSON list of {"case", "bar", "errors"}).
PARITY_RECORD: list = []


def record(case: str, errs: dict, bar: float) -> None:
    PARITY_RECORD.append({"case": case, "bar": bar, "errors": {k: float(v) for k, v in errs.items()}})
    print(case, {k: f"{v:.2e}" for k, v in errs.items()})
