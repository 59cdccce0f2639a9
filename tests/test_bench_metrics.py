"""The ground-truth parameter error that bench.py reports (param_error): its
Euler -> quaternion -> normal chain agrees with the oracle's Euler matrix (the
reference's convention), the true parameters of synthetic texels score zero
error, and known perturbations score what they should."""
import numpy as np

import bench
import oracle


def _truths(n, seed=31, mix=1):
    rows = []
    for x in range(n):
        t = oracle.synth_truth(seed, mix, x)
        rows.append([*t.kd[:], *t.ks[:], *t.sigma[:], *t.quat[:], *t.euler[:], float(t.kind)])
    return np.array(rows, np.float64)


def test_normal_of_euler_matches_the_oracle_matrix():
    rng = np.random.default_rng(3)
    e = rng.uniform(-np.pi, np.pi, (64, 3))
    n = bench._normal_of_quat(bench._quat_of_euler(e))
    for k in range(len(e)):
        R, _ = oracle.euler_to_matrix(e[k])   # R[c] is column c; column 2 is the normal
        np.testing.assert_allclose(np.abs(n[k] @ np.asarray(R[2], np.float64)), 1.0, atol=1e-6)


def test_true_parameters_score_zero_error():
    tr = _truths(200)
    params = np.stack([oracle.truth_lum_params(oracle.synth_truth(31, 1, x)) for x in range(len(tr))])
    err = bench.param_error(params, tr)
    assert err["normal_deg"]["p90"] < 0.05, err
    for k in ("log_scale", "log_anisotropy", "kd_rel", "ks_rel"):
        assert err[k]["p90"] < 1e-5, (k, err[k])


def test_perturbations_score_what_they_should():
    tr = _truths(100)
    p = np.stack([oracle.truth_lum_params(oracle.synth_truth(31, 1, x)) for x in range(len(tr))]).astype(np.float64)
    # both scales x 1.1: |log| of the geometric-mean scale is log 1.1, the anisotropy unchanged
    q = p.copy()
    q[:, 0:2] *= 1.1
    err = bench.param_error(q, tr)
    assert abs(err["log_scale"]["median"] - np.log(1.1)) < 1e-5
    assert err["log_anisotropy"]["p90"] < 1e-5
    # albedos + 10 % (where the truth is above the 0.02 floor): relative error 0.1
    q = p.copy()
    q[:, 2:4] *= 1.1
    err = bench.param_error(q, tr)
    assert abs(err["kd_rel"]["median"] - 0.1) < 1e-3 and abs(err["ks_rel"]["median"] - 0.1) < 1e-3
    # the true frame turned by 2 degrees about its tangent (q -> q (x) r, r = rotation about local x):
    # the normal of the fitted (true) Euler angles is then 2 degrees off
    th = np.radians(2.0)
    sn, cs = np.sin(th / 2), np.cos(th / 2)
    x1, y1, z1, w1 = tr[:, 8], tr[:, 9], tr[:, 10], tr[:, 11]
    t2 = tr.copy()
    t2[:, 8:12] = np.stack([w1 * sn + x1 * cs, y1 * cs + z1 * sn, z1 * cs - y1 * sn, w1 * cs - x1 * sn], 1)
    err = bench.param_error(p, t2)
    assert abs(err["normal_deg"]["median"] - 2.0) < 0.01 and abs(err["normal_deg"]["p90"] - 2.0) < 0.01, err
