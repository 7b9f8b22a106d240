"""Vina-potential tables (ag_job_vina_problem) against an independent numpy
restatement of main.cpp:2081-2126 with the xs radii of
read_parameter_library.cc:323-339, on the CPU.  The reference compiles this
path out (use_vina_potential = FALSE, main.cpp:263) and has no test for it, so
parity with the reference's own output is unpinned; this pins the engine to
the reference source as written.
"""
import numpy as np
import pytest

from conftest import make_case

XS = {"C": 1.9, "A": 1.9, "N": 1.8, "NA": 1.8, "NS": 1.8, "O": 1.7, "OA": 1.7, "OS": 1.7, "S": 2.0,
      "SA": 2.0, "P": 2.1, "F": 1.5, "Mg": 1.2}
W = dict(g1=-0.035579, g2=-0.005156, rep=0.840245, h=-0.587439, hp=-0.035069)


def _gpf_types(path):
    rec, lig = None, None
    for line in open(path):
        f = line.split()
        if f and f[0] == "receptor_types":
            rec = f[1:]
        if f and f[0] == "ligand_types":
            lig = f[1:]
    return rec, lig


def _hbonder(mh, rh):
    return int(((mh > 2 or mh == 6) and rh in (1, 2, 6)) or (mh in (1, 2, 6) and rh > 2))


def _restated(rec_types, lig_types, map_hbond, rec_hbond):
    f32 = np.float32
    w = {k: float(f32(v)) for k, v in W.items()}
    nR, nAM = len(rec_types), len(lig_types)
    tab = np.zeros((nR, nAM, 1024), dtype=np.float32)
    hb = [[_hbonder(map_hbond[ia], rec_hbond[i]) for i in range(nR)] for ia in range(nAM)]
    r = np.arange(1, 1024) / 128.0
    for ia in range(nAM):
        Rij = float(f32(XS.get(lig_types[ia], 1.8)))
        for i in range(nR):
            mR = float(f32(XS.get(rec_types[i], 1.8)))
            d = r - (mR + Rij)
            t = np.zeros(1023, dtype=np.float32)
            t = (t.astype(np.float64) + w["g1"] * np.exp(-(d / 0.5) ** 2) + w["g2"] * np.exp(-((d - 3.0) / 2.0) ** 2)).astype(np.float32)
            t = np.where(d < 0, (t.astype(np.float64) + w["rep"] * d ** 2).astype(np.float32), t)
            if hb[ia][i] > 0:
                t = np.where(d <= 0.7, (t.astype(np.float64) + w["h"]).astype(np.float32), t)
                t = np.where((-0.7 < d) & (d <= 0.0), (t.astype(np.float64) - (d / 0.7) * w["h"]).astype(np.float32), t)
            # gridmap[i].hbonder[ia]: zero for the e/d map objects and past the receptor types
            alias = hb[i][ia] if (i < nAM and ia < nR) else 0
            if hb[ia][i] == 0 and alias == 0:
                de = np.where(d < 0.5, w["hp"], np.where(d < 1.5, (0.5 - d) * w["hp"], 0.0))
                t = (t.astype(np.float64) + de).astype(np.float32)
            tab[i, ia, 1:] = t
    return tab


@pytest.mark.parametrize("ligands", [["A", "C", "F", "HD", "N", "NA", "OA", "SA"], ["C", "OA", "HD", "Cl", "S"]])
def test_vina_tables_match_restatement(tmp_path, built, ligands):
    job, prob = make_case(tmp_path, "v", 600, (10, 10, 10), seed=2, radius=12.0, ligand_types=ligands)
    vp = job.vina_problem()
    rec_types, lig_types = _gpf_types(tmp_path / "v.gpf")
    assert lig_types == ligands
    assert vp.n_maps == len(ligands) and vp.scalars["elec_map"] == -1 and vp.scalars["dsolv_map"] == -1
    assert not vp.arrays["map_is_hbonder"].any() and not vp.arrays["map_solpar_probe"].any()
    # receptor hbond class per receptor type, from the atoms
    rec_hbond = [int(prob.arrays["hbond"][np.flatnonzero(prob.arrays["rec_type"] == i)[0]]) for i in range(len(rec_types))]
    want = _restated(rec_types, lig_types, prob.arrays["map_hbond"], rec_hbond)
    got = vp.arrays["e_vdw_hb"].reshape(want.shape)
    assert np.array_equal(got, want), np.abs(got - want).max()
    # the AD4 problem of the same job is untouched
    assert np.array_equal(job.problem().arrays["e_vdw_hb"], prob.arrays["e_vdw_hb"])
