"""The cheaper propagation forms in the two Earth-fixed frames, in the oracle
(CPU): DOP853 at eps 1e-10 and Vern9 at eps 1e-10 against DOP853 at eps 1e-12
on 8 of the bench's LEO rows (70x70 + JB2008 + Sun/Moon), over one day by
default (``BQP_FORMS_DAYS=7`` for the week of the accuracy bound; ``-s``
prints the table).

The GMST frame's 40 us time staircase inflates the eps 1e-12 reference run
(it drives the step controller) but not the eps 1e-10 forms, so the forms'
evaluation ratio against the reference is smaller in the GMST frame than in
the IAU frame, which is the reference's production frame."""
import os

import numpy as np

from bqp_b200 import _native as N
from bqp_b200 import workloads
from oracle import oracle as O

FORMS = (("dop853 eps 1e-12", "dop853", 1e-12), ("dop853 eps 1e-10", "dop853", 1e-10),
         ("vern9 eps 1e-10", "vern9", 1e-10))


def run(days):
    n = 8
    text = workloads.synthetic_field(70)
    states = workloads.leo_states(65536, seed=0)[::65536 // n]
    bal = workloads.leo_ballistics(65536, seed=0)[::65536 // n]
    equ = np.array([O.eci2equinoc(s)[0] for s in states])
    epoch = workloads.EPOCH_JD
    tf = days * 86400.0
    F = O.Force(text, 70, drag=True, sun=True, moon=True)
    auth = N.FrameAuthority()
    tai0 = N.tai_seconds(epoch)[0]
    keys, segs = auth.segments(tai0 - 1800.0, tai0 + tf + 1800.0)
    out = {}
    for frame in ("gmst", "iau2006"):
        if frame == "iau2006":
            F.set_frame(keys, segs, auth.intervals()["raw"])
        else:
            F.set_frame()
        for name, method, eps in FORMS:
            d, st, _, ev = O.propagate_final_batch(F, O.ctrl(method, eps=eps), equ, epoch, tf, bal, threads=0)
            assert (st == 0).all(), (frame, name, st)
            pos = np.array([O.equinoc2eci(equ[i], tf)[0][:3] + d[i][:3] for i in range(n)])
            out[(frame, name)] = (pos, float(ev.sum()))
    return out


def test_forms_in_both_frames():
    days = float(os.environ.get("BQP_FORMS_DAYS", "1"))
    out = run(days)
    ratio = {}
    for frame in ("gmst", "iau2006"):
        ref_pos, ref_ev = out[(frame, FORMS[0][0])]
        for name, _, _ in FORMS[1:]:
            pos, ev = out[(frame, name)]
            err_m = float(np.linalg.norm(pos - ref_pos, axis=1).max() * 1000.0)
            ratio[(frame, name)] = ev / ref_ev
            print(f"{frame:8s} {name:17s} {days:g} d: max |dr| {err_m:.4f} m, evaluations x{ev / ref_ev:.3f}")
            assert err_m <= 1.0  # the metric's bound
    # the eps 1e-12 reference costs less in the IAU frame, the eps 1e-10
    # forms the same in both
    assert out[("iau2006", FORMS[0][0])][1] < 0.8 * out[("gmst", FORMS[0][0])][1]
    for name, _, _ in FORMS[1:]:
        a, b = out[("gmst", name)][1], out[("iau2006", name)][1]
        assert abs(a - b) <= 0.05 * a
        assert ratio[("iau2006", name)] > ratio[("gmst", name)]
