"""Every device-side wait of the flag-synchronised BILU(0) kernels is bounded.

The flag-scheduled factor and sweeps (kernel/computeBILU0.m and kernel/applyBILU0.m in a
sequential order, rows taken through a work counter) wait for the ready flags of the rows
they depend on.  Here a schedule is built whose flag is never set: the work list names one
row twice and leaves out the first row of the minimum-discarded-fill order, so the rows
coupled to it wait for a flag that nothing writes.  With a small poll limit (sched[3]) each
such wait runs out, raises the error flag and lets its row go on; hdgx_gmres_bilu0 then
returns status -14 (the reference's solver reports failures through its flags output,
kernel/gmres_bilu0.m:78-91).  Every index in that schedule is a valid row, so nothing reads
or writes out of bounds.  The context stays usable: the same system is solved afterwards
with the valid order."""
import numpy as np
import pytest

from hdg_b200 import configs


@pytest.mark.gpu
def test_flag_wait_runs_out_reports_and_leaves_the_gpu_usable(oracle):
    from hdg_b200._lib import HdgxError
    from hdg_b200.elemental import DArray
    from hdg_b200.solve import TraceSystem
    P = configs.c1(n=4, porder=2)
    r = oracle.hdg_elemental(P.master, P.app, P.mesh.dgnodes, P.mesh.bf, P.UDG, P.uh_elem(), P.SH)
    Hg, Rg = oracle.globalassembly(P.mesh, r["AE"], r["FE"], P.master.npf, P.app.ncu)
    ts = TraceSystem(P.mesh, P.master, P.app, ordering="mdf")
    dH, dR = DArray.from_numpy(Hg), DArray.from_numpy(Rg)
    o2u, u2o = ts.mdf_order(dH)
    # the first row of the order is never processed; the second is listed twice
    bad = o2u.copy()
    bad[0] = o2u[1]
    first = int(o2u[0])
    rp = P.mesh.cbsr_rowpts
    assert rp[first + 1] - rp[first] > 1                 # some rows are coupled to it
    ts.set_order(bad, u2o)
    ts.sched[3] = 2000                                   # poll limit of every wait
    dM = ts.empty_blocks()
    ts.bilu0(dH, dM)
    x = ts.empty_vec()
    x.t.zero_()
    with pytest.raises(HdgxError) as e:
        ts.gmres(dH, dM, dR, x, restart=20, tol=1e-10, maxit=4)
    assert "status -14" in str(e.value)
    assert int(ts.sched[2].item()) == 0                  # the error flag is cleared for the next call
    # the GPU and the context are still usable: the valid schedule solves the system
    ts.set_order(o2u, u2o)
    ts.bilu0(dH, dM)
    x.t.zero_()
    it, fl, rr, _ = ts.gmres(dH, dM, dR, x, restart=20, tol=1e-10, maxit=500)
    assert fl == 0 and rr <= 1e-10
    assert np.isfinite(x.numpy()).all()
