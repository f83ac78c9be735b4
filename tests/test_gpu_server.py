"""The serving layer (hdd_server_*): concurrent solves of uneven domains.

* every request's iterations and solution equal the plain one-handle solve of
  the same domain and right-hand side, bit for bit, whether it ran alone or
  among other requests in flight, on the same domain (several solve contexts
  of one resident domain at once) or on others;
* a budget that fits one domain at a time admits them in turn and all
  requests still finish; the reserved bytes return to zero after removal;
* a domain whose setup fails reports its status, and so do its requests.
"""
import numpy as np
import pytest

from hierarchicaldd_b200 import domains
from hierarchicaldd_b200._lib import HddError
from hierarchicaldd_b200.server import SolveServer, make_options

pytestmark = pytest.mark.gpu


def cases():
    return [domains.small(32, 8, 6, seed=1), domains.small((40, 36, 44), 8, 6, seed=11),
            domains.small(48, 16, 8, seed=7), domains.small(16, 16, 3, seed=1)]


def options(d, **extra):
    m = d.meta
    return make_options(d.size, d.sub_size, m["vlevels"], m["nVcycles"], m["interior_smoothing"],
                        m["boundary_smoothing"], m["sigma_levels"], m["sigma_smoothing"], m["sigma_mg"], **extra)


def rhs_set(d, k):
    rng = np.random.Generator(np.random.Philox(100 + k))
    out = [d.rhs]
    for _ in range(k):
        r = rng.uniform(-1, 1, d.size).astype(np.float32)
        r[(d.flags & domains.ACTIVE) == 0] = 0
        out.append(r)
    return out


def solo(d, rhs_list):
    from hierarchicaldd_b200.solver import SPGrid_Domain_Decomposition_Solver
    m = d.meta
    s = SPGrid_Domain_Decomposition_Solver()
    s.Set_Domain(d.flags, d.rhs)
    s.Initialize_Preconditioner(m["vlevels"], d.size, d.sub_size, m["sigma_levels"], m["nVcycles"],
                                m["interior_smoothing"], m["boundary_smoothing"], m["sigma_smoothing"], m["sigma_mg"])
    out = []
    for r in rhs_list:
        s.Set_RHS(r)
        res = s.Solve()
        out.append((res["iterations"], s.Solution()))
    s.close()
    return out


def test_concurrent_requests_match_plain_solves():
    ds = cases()
    rhs = [rhs_set(d, 2) for d in ds]
    ref = [solo(d, r) for d, r in zip(ds, rhs)]
    srv = SolveServer(slots=3)
    try:
        ids = [srv.add_domain(d.flags, options(d)) for d in ds]
        # Alone: one request at a time on the resident domains.
        for i, dom in enumerate(ids):
            assert srv.wait_domain(dom)
            req = srv.submit(dom, rhs[i][0])
            st, res, x, lat = srv.poll(req, dom)
            assert st == 0 and res["converged"] == 1 and lat > 0
            assert res["iterations"] == ref[i][0][0] and np.array_equal(x, ref[i][0][1])
        # In the mix: every request submitted at once, interleaved over domains.
        reqs = [(i, k, srv.submit(ids[i], rhs[i][k])) for k in range(3) for i in range(len(ds))]
        for i, k, req in reqs:
            st, res, x, _ = srv.poll(req, ids[i])
            assert st == 0, (i, k, st)
            assert res["iterations"] == ref[i][k][0], (i, k)
            assert np.array_equal(x, ref[i][k][1]), (i, k, float(np.max(np.abs(x - ref[i][k][1]))))
        for dom in ids:
            srv.remove_domain(dom)
        assert srv.memory()[0] == 0
    finally:
        srv.close()


def test_one_domain_many_requests_in_flight():
    # Six requests on one domain with four slots: up to four solve contexts of
    # the domain run at once (precision form, exact coarsest interface level).
    d = domains.small(48, 16, 8, seed=7)
    m = d.meta
    rhs = rhs_set(d, 5)
    from hierarchicaldd_b200.solver import SPGrid_Domain_Decomposition_Solver
    s = SPGrid_Domain_Decomposition_Solver()
    s.Set_Domain(d.flags, d.rhs)
    s.Initialize_Preconditioner(m["vlevels"], d.size, d.sub_size, m["sigma_levels"], m["nVcycles"],
                                m["interior_smoothing"], m["boundary_smoothing"], m["sigma_smoothing"], m["sigma_mg"],
                                precision_mode=1, true_residual_every=20)
    ref = []
    for r in rhs:
        s.Set_RHS(r)
        res = s.Solve()
        ref.append((res["iterations"], s.Solution()))
    s.close()
    srv = SolveServer(slots=4)
    try:
        dom = srv.add_domain(d.flags, options(d, precision_mode=1, true_residual_every=20))
        assert srv.wait_domain(dom)
        one = srv.memory()[0]
        for rnd in range(2):
            reqs = [srv.submit(dom, r) for r in rhs]
            for k, req in enumerate(reqs):
                st, res, x, _ = srv.poll(req, dom)
                assert st == 0, (rnd, k, st)
                assert res["iterations"] == ref[k][0], (rnd, k)
                assert np.array_equal(x, ref[k][1]), (rnd, k, float(np.max(np.abs(x - ref[k][1]))))
        # Contexts beyond the first are counted against the budget.
        assert srv.memory()[0] >= one
        srv.remove_domain(dom)
        assert srv.memory()[0] == 0
    finally:
        srv.close()


def test_solve_share_does_not_change_results():
    # The persistent interface solves on a fraction of the device: the same
    # tasks in the same order on fewer CTAs, so the same bits.
    from hierarchicaldd_b200.solver import SPGrid_Domain_Decomposition_Solver
    d = domains.small(64, 16, 10, seed=3)
    m = d.meta
    out = []
    for share in (0, 2, 7):
        s = SPGrid_Domain_Decomposition_Solver()
        s.Set_Domain(d.flags, d.rhs)
        s.Initialize_Preconditioner(m["vlevels"], d.size, d.sub_size, m["sigma_levels"], m["nVcycles"],
                                    m["interior_smoothing"], m["boundary_smoothing"], m["sigma_smoothing"],
                                    m["sigma_mg"], solve_share=share)
        res = s.Solve()
        out.append((res["iterations"], s.Solution()))
        s.close()
    for its, x in out[1:]:
        assert its == out[0][0] and np.array_equal(x, out[0][1])


def test_budget_admits_domains_in_turn():
    ds = cases()[:3]
    probe = SolveServer(slots=1)
    try:
        sizes = []
        for d in ds:
            dom = probe.add_domain(d.flags, options(d))
            sizes.append(probe.memory()[0])  # the estimate, or the actual if set up already
            assert probe.wait_domain(dom)
            sizes.append(probe.memory()[0])  # what the solver holds
            probe.remove_domain(dom)
    finally:
        probe.close()
    srv = SolveServer(slots=2, hbm_budget_bytes=int(max(sizes) * 1.05))
    try:
        ids = [srv.add_domain(d.flags, options(d)) for d in ds]
        reqs = [(i, srv.submit(dom, d.rhs)) for i, (dom, d) in enumerate(zip(ids, ds))]
        # Later domains wait for budget until earlier ones are removed.
        for i, req in reqs:
            st, res, _, _ = srv.poll(req, ids[i], want_x=False)
            assert st == 0 and res["converged"] == 1
            srv.remove_domain(ids[i])
        assert srv.memory()[0] == 0
    finally:
        srv.close()


def test_failed_domain_reports_its_status():
    d = domains.small(16, 8, 0, seed=1)
    d.flags[:] = 0
    srv = SolveServer(slots=2)
    try:
        dom = srv.add_domain(d.flags, options(d))
        req = srv.submit(dom, np.zeros(d.size, np.float32))
        with pytest.raises(HddError) as e:
            srv.wait_domain(dom)
        assert e.value.status == 1 and "no Active cells" in str(e.value)
        st, _, _, _ = srv.poll(req, dom, want_x=False)
        assert st == 1
        srv.remove_domain(dom)
    finally:
        srv.close()


@pytest.mark.parametrize("batch,precision", [(4, 0), (2, 1), (4, 1)])
def test_batched_requests_equal_solo_solves(batch, precision):
    # Continuous batching: a domain's requests solved k at a time in shared
    # launches (multi-right-hand-side interface solves, V-cycles over all
    # systems), requests joining as systems free up.  Every result equals the
    # request's solve alone, bit for bit.
    ds = [domains.small(48, 16, 8, seed=7), domains.small((40, 36, 44), 8, 6, seed=11)]
    rhs = [rhs_set(d, 6) for d in ds]
    from hierarchicaldd_b200.solver import SPGrid_Domain_Decomposition_Solver
    ref = []
    for d, rl in zip(ds, rhs):
        m = d.meta
        s = SPGrid_Domain_Decomposition_Solver()
        s.Set_Domain(d.flags, d.rhs)
        s.Initialize_Preconditioner(m["vlevels"], d.size, d.sub_size, m["sigma_levels"], m["nVcycles"],
                                    m["interior_smoothing"], m["boundary_smoothing"], m["sigma_smoothing"],
                                    m["sigma_mg"], precision_mode=precision, true_residual_every=5)
        out = []
        for r in rl:
            s.Set_RHS(r)
            res = s.Solve()
            out.append((res["iterations"], s.Solution()))
        s.close()
        ref.append(out)
    srv = SolveServer(slots=2, batch=batch)
    try:
        ids = [srv.add_domain(d.flags, options(d, precision_mode=precision, true_residual_every=5)) for d in ds]
        for dom in ids:
            assert srv.wait_domain(dom)
        # All at once, interleaved over the two domains; then a second wave
        # submitted while the first is still being solved.
        reqs = [(i, k, srv.submit(ids[i], rhs[i][k])) for k in range(4) for i in range(len(ds))]
        reqs += [(i, k, srv.submit(ids[i], rhs[i][k])) for k in range(4, 7) for i in range(len(ds))]
        for i, k, req in reqs:
            st, res, x, _ = srv.poll(req, ids[i])
            assert st == 0, (i, k, st)
            assert res["iterations"] == ref[i][k][0], (i, k, res["iterations"], ref[i][k][0])
            assert np.array_equal(x, ref[i][k][1]), (i, k, float(np.max(np.abs(x - ref[i][k][1]))))
        for dom in ids:
            srv.remove_domain(dom)
        assert srv.memory()[0] == 0
    finally:
        srv.close()
