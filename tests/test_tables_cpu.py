"""The table parameters a job exports (ag_job_table_params) rebuild the job's
own tables exactly, through a plain-Python restatement of main.cpp:2040-2276
(LJ/H-bond pair tables with clamp and +-smooth/2 minimum filter, desolvation
table) and distdepdiel.cpp:30-57 (Mehler-Solmajer), using the host libm's pow
and exp as the front end does.  This pins the inputs that ag_tables_build
(the device table build) consumes."""
import math

import numpy as np
import pytest

from test_oracle_pinning import GOLDEN, load_golden

NEINT, NDIEL, A_DIV = 1024, 8192, 128
EINTCLAMP = 100000.0


def _arr(ptr, n):
    return np.ctypeslib.as_array(ptr, shape=(n,)).copy() if n else np.zeros(0)


def restate(tp):
    nT, nAM = tp.n_rec_types, tp.n_atom_maps
    n = nT * nAM
    cA_, cB_ = _arr(tp.cA, n), _arr(tp.cB, n)
    R_, E_ = _arr(tp.Rij, n), _arr(tp.epsij, n)
    xA_, xB_ = _arr(tp.xA, n), _arr(tp.xB, n)
    cov = _arr(tp.map_is_covalent, nAM)
    tab = np.zeros((nT, nAM, NEINT), dtype=np.float32)
    i_smooth = int(tp.r_smooth * A_DIV / 2.0)
    for m in range(nAM):
        if cov[m]:
            continue
        for t in range(nT):
            k = m * nT + t
            cA, cB, xA, xB = float(cA_[k]), float(cB_[k]), int(xA_[k]), int(xB_[k])
            if cA == 0 and cB == 0:
                tmp = float(E_[k]) / float(xA - xB)
                cA = tmp * math.pow(float(R_[k]), float(xA)) * float(xB)
                cB = tmp * math.pow(float(R_[k]), float(xB)) * float(xA)
            row = np.empty(NEINT, dtype=np.float32)
            for b in range(1, NEINT):
                r = float(b) * (1.0 / A_DIV)
                v = cA / math.pow(r, float(xA)) - cB / math.pow(r, float(xB))
                row[b] = np.float32(EINTCLAMP if EINTCLAMP < v else v)
            row[0] = np.float32(EINTCLAMP)
            row[NEINT - 1] = 0.0
            if i_smooth > 0:
                sm = np.empty(NEINT, dtype=np.float32)
                for b in range(NEINT):
                    lo, hi = max(0, b - i_smooth), min(NEINT, b + i_smooth + 1)
                    sm[b] = np.float32(min(100000.0, float(row[lo:hi].astype(np.float64).min())))
                row = sm
            tab[t, m] = row
    sol = np.zeros(NDIEL)
    for b in range(1, NDIEL):
        r = float(b) * (1.0 / A_DIV)
        sol[b] = tp.coeff_desolv * math.exp(-(r * r) / (2.0 * (3.6 * 3.6)))
    eps = None
    if tp.dddiel:
        lam, e0, A, rk = 0.003627, 78.4, -8.5525, 7.7839
        B = e0 - A
        eps = np.zeros(NDIEL)
        for b in range(NDIEL):
            if b == 0:
                e = 1.0
            else:
                r = float(b) * (1.0 / A_DIV)
                e = A + B / (1.0 + rk * math.exp(-lam * B * r))
                if e < 1e-6:
                    e = 1.0
            eps[b] = 332.0 / e
    return tab, sol, eps


@pytest.mark.parametrize("path", [p for p in GOLDEN if p.stem in ("basic_400", "constdiel_nbp", "disorder_sep_cov")],
                         ids=lambda p: p.stem)
def test_table_params_rebuild_job_tables(path, tmp_path):
    _, job, prob = load_golden(path, tmp_path)
    tp = job.table_params()
    tab, sol, eps = restate(tp)
    np.testing.assert_array_equal(tab.reshape(-1), prob.arrays["e_vdw_hb"][: tab.size])
    np.testing.assert_array_equal(sol, prob.arrays["sol_fn"][:NDIEL])
    if eps is not None:
        np.testing.assert_array_equal(eps, prob.arrays["r_epsilon_fn"][:NDIEL])
    job.close()
