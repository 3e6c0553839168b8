"""Serving loop (tg_server_*): a request's result does not depend on what else is resident
(alone == mixed, bit for bit, and == tg_step on a lone context), admission respects the HBM
budget, and failures (over budget, non-finite energy, bad configuration) stay with the request
that caused them."""

import math

import numpy as np
import pytest

from oracle import tarang_oracle as o
from tarang_b200 import _lib as L
from tarang_b200 import ic

pytestmark = pytest.mark.gpu

KF = (1.0, 1.0, 1.0)
KF_RB = (math.pi, math.pi / math.sqrt(2.0), math.pi / math.sqrt(2.0))


def fluid_fields(N, seed, energy=1.0):
    return ic.random_phase_field(N, seed=seed, energy=energy)


def mhd_fields(N, seed):
    return ic.random_phase_field(N, seed=seed) + ic.random_phase_field(N, seed=seed + 1, energy=0.5)


def rb_fields(N, seed):
    """SCFT fields: u1 and theta sine series, u2 and u3 cosine series (dealiased)."""
    rng = np.random.default_rng(seed)
    return [1e-2 * o.dealias(o.forward_scft(rng.standard_normal(N), p), "SCFT") for p in (1, 0, 0, 1)]


def lone(config, fields, n):
    from tarang_b200.solver import IncFluid
    cfg = dict(config)
    N = cfg.pop("N")
    s = IncFluid(N, **cfg)
    s.set_V(fields[:3])
    if len(fields) == 6:
        s.set_W(fields[3:])
    elif len(fields) == 4:
        s.set_T(fields[3])
    s.step(n)
    out = s.get_V()
    if len(fields) == 6:
        out += s.get_W()
    elif len(fields) == 4:
        out.append(s.get_T())
    t, steps = s.time()
    s.close()
    return out, t, steps


def same_bits(a, b):
    return all(np.array_equal(x.view(np.float64), y.view(np.float64)) for x, y in zip(a, b))


def run_alone(config, fields, n, **kw):
    from tarang_b200.serving import Server
    with Server(hbm_budget=kw.pop("hbm_budget", 8e9), **kw) as srv:
        rid = srv.submit(config, fields, n)
        srv.drain()
        st = srv.poll(rid)
        assert st["state"] == "done", st
        return srv.result(rid), st


X_CFG = dict(N=(32, 32, 32), nu=3e-3, dt=2e-3)


def mixed_population(n_steps):
    """(config, fields, steps) of a mixed load: same shape with other coefficients and step
    counts, other shapes, MHD, FP32, SCFT Rayleigh-Benard."""
    pop = []
    for j, nu in enumerate([1e-3, 5e-3, 1e-2]):
        pop.append((dict(N=(32, 32, 32), nu=nu, dt=1e-3 * (j + 1)), fluid_fields((32, 32, 32), 100 + j), n_steps - 3 + 2 * j))
    pop.append((dict(N=(16, 16, 32), nu=2e-3, dt=1e-3), fluid_fields((16, 16, 32), 200), n_steps + 4))
    pop.append((dict(N=(16, 16, 16), physics="MHD", nu=2e-3, eta=4e-3, dt=1e-3), mhd_fields((16, 16, 16), 300), n_steps))
    pop.append((dict(N=(32, 32, 32), nu=2e-3, dt=1e-3, precision="FP32"), fluid_fields((32, 32, 32), 400), n_steps))
    pop.append((dict(N=(17, 16, 32), basis="SCFT", physics="RB", Ra=2e4, Pr=1.0, dt=1e-3, kfactor=KF_RB),
                rb_fields((17, 16, 32), 500), n_steps))
    return pop


def test_alone_equals_lone_context(lib):
    X = fluid_fields(X_CFG["N"], 7)
    got, st = run_alone(X_CFG, X, 12)
    want, t, steps = lone(X_CFG, X, 12)
    assert same_bits(got, want)
    assert st["steps_done"] == 12 and steps == 12 and st["t_final"] == t


@pytest.mark.parametrize("use_graphs", [True, False])
def test_alone_equals_mixed(lib, use_graphs):
    from tarang_b200.serving import Server
    n = 10
    X = fluid_fields(X_CFG["N"], 7)
    alone, _ = run_alone(X_CFG, X, n, use_graphs=use_graphs)
    pop = mixed_population(n)
    with Server(hbm_budget=8e9, max_batch=8, use_graphs=use_graphs) as srv:
        ids = [srv.submit(c, f, k) for c, f, k in pop[:3]]
        xid = srv.submit(X_CFG, X, n)
        ids += [srv.submit(c, f, k) for c, f, k in pop[3:]]
        srv.drain()
        mixed = srv.result(xid)
        assert same_bits(mixed, alone)
        # every other request equals its lone-context run as well
        for rid, (c, f, k) in zip(ids, pop):
            st = srv.poll(rid)
            assert st["state"] == "done" and st["steps_done"] == k
            want, _, _ = lone(c, f, k)
            assert same_bits(srv.result(rid), want), c
        s = srv.stats()
        assert s["request_steps"] == n + sum(k for _, _, k in pop)
        if use_graphs:
            assert s["graph_launches"] > 0


def test_late_arrivals_join_running_batch(lib):
    """Requests submitted between pumps join the running batch of their shape; slots move as
    requests leave; every result equals its lone run."""
    from tarang_b200.serving import Server
    N = (32, 32, 32)
    reqs = [(dict(N=N, nu=1e-3 * (1 + j), dt=1e-3), fluid_fields(N, 600 + j), 4 + 3 * (j % 3)) for j in range(7)]
    with Server(hbm_budget=8e9, max_batch=4) as srv:
        ids = []
        for j, (c, f, k) in enumerate(reqs):
            ids.append(srv.submit(c, f, k))
            srv.pump()
            if j % 2:
                srv.pump()
        srv.drain()
        for rid, (c, f, k) in zip(ids, reqs):
            want, _, _ = lone(c, f, k)
            assert same_bits(srv.result(rid), want)


def test_split_pump_submits_during_round(lib):
    """pump_begin / submit / pump_end: requests submitted while a round runs on the device are
    admitted at its end and join the running batch; a second pump_begin on an open round is
    TG_ERR_STATE; drain closes an open round; every result equals its lone run."""
    from tarang_b200.serving import Server
    N = (32, 32, 32)
    reqs = [(dict(N=N, nu=1e-3 * (1 + j), dt=1e-3), fluid_fields(N, 800 + j), 3 + 2 * (j % 3)) for j in range(6)]
    with Server(hbm_budget=8e9, max_batch=4) as srv:
        ids = [srv.submit(*reqs[0])]
        srv.pump()
        for j in range(1, len(reqs)):
            srv.pump_begin()
            if j == 1:
                with pytest.raises(L.TarangError) as e:
                    srv.pump_begin()
                assert e.value.code == L.TG_ERR_STATE
            ids.append(srv.submit(*reqs[j]))
            assert srv.poll(ids[-1])["state"] == "queued"
            srv.pump_end()
            assert srv.poll(ids[-1])["state"] in ("running", "done")
        srv.pump_begin()
        srv.drain()
        assert srv.pump_end() == 0          # admission-only round on an empty server
        for rid, (c, f, k) in zip(ids, reqs):
            want, _, _ = lone(c, f, k)
            assert same_bits(srv.result(rid), want)


def test_borrowed_inputs(lib):
    """borrow_inputs: submit keeps the caller's arrays (no copy) and admission reads them; the
    results equal those of copied inputs bit for bit, and the caller may reuse an array once its
    request runs."""
    from tarang_b200.serving import Server
    N = (32, 32, 32)
    cfgs = [dict(N=N, nu=1e-3 * (1 + j), dt=1e-3) for j in range(4)]
    fields = [np.ascontiguousarray(np.stack(fluid_fields(N, 900 + j))) for j in range(4)]
    with Server(hbm_budget=8e9, max_batch=4) as a, Server(hbm_budget=8e9, max_batch=4, borrow_inputs=True) as b:
        ia = [a.submit(c, f, 5) for c, f in zip(cfgs, fields)]
        ib = [b.submit(c, f, 5) for c, f in zip(cfgs, fields)]
        assert len(b._held) == 4
        b.pump()
        assert not b._held and all(b.poll(i)["state"] != "queued" for i in ib)
        kept = [f.copy() for f in fields]
        for f in fields:
            f[...] = 0          # the requests run: their inputs are no longer read
        a.drain()
        b.drain()
        for x, y, f in zip(ia, ib, kept):
            assert same_bits(a.result(x), b.result(y))
            want, _, _ = lone(cfgs[0] if x == ia[0] else cfgs[ia.index(x)], list(f), 5)
            assert same_bits(b.result(y), want)


def test_budget_admission(lib):
    from tarang_b200.serving import Server, request_bytes
    cfg = dict(N=(32, 32, 32), nu=2e-3, dt=1e-3)
    one = request_bytes(cfg, 1)
    budget = int(one * 1.5)        # room for one request at a time
    reqs = [fluid_fields((32, 32, 32), 700 + j) for j in range(3)]
    with Server(hbm_budget=budget, max_batch=8) as srv:
        ids = [srv.submit(cfg, f, 5) for f in reqs]
        srv.pump()
        s = srv.stats()
        assert s["n_running"] == 1 and s["n_queued"] == 2
        assert s["bytes_resident"] == one
        srv.drain()
        s = srv.stats()
        assert s["bytes_peak"] <= budget and s["n_running"] == 0 and s["n_queued"] == 0
        assert s["n_batches"] == 1     # the idle batch stays resident for the next request
        starts = sorted(srv.poll(i)["start_s"] for i in ids)
        finishes = sorted(srv.poll(i)["finish_s"] for i in ids)
        assert starts[1] >= finishes[0] and starts[2] >= finishes[1]
        assert sorted(srv.take_finished()) == sorted(ids) and srv.take_finished() == []
        for rid, f in zip(ids, reqs):
            want, _, _ = lone(cfg, f, 5)
            assert same_bits(srv.result(rid), want)


def test_request_bytes_match_allocation(lib):
    from tarang_b200.serving import request_bytes
    from tarang_b200.solver import IncFluid
    for cfg in [dict(N=(32, 32, 32)), dict(N=(16, 16, 32), physics="MHD"), dict(N=(32, 32, 32), precision="FP32"),
                dict(N=(17, 16, 32), basis="SCFT", physics="RB", Ra=1e4, Pr=1.0),
                dict(N=(32, 32, 32), force=dict(inner=2.0, outer=3.0, eps=0.1))]:
        c = dict(cfg)
        N = c.pop("N")
        s = IncFluid(N, **c)
        s.set_V(fluid_fields(N, 1))
        s.get_V()                        # the whole-array download allocates the dense staging field
        assert s.device_bytes() == request_bytes(cfg, 1), cfg
        s.close()


def test_over_budget_request_fails_alone(lib):
    from tarang_b200.serving import Server, request_bytes
    small = dict(N=(16, 16, 16), nu=2e-3, dt=1e-3)
    big = dict(N=(64, 64, 64), nu=2e-3, dt=1e-3)
    budget = request_bytes(small, 1) * 3
    assert request_bytes(big, 1) > budget
    with Server(hbm_budget=budget) as srv:
        a = srv.submit(small, fluid_fields((16, 16, 16), 1), 3)
        b = srv.submit(big, fluid_fields((64, 64, 64), 2), 3)
        st = srv.poll(b)
        assert st["state"] == "failed" and st["error"] == L.TG_ERR_OOM
        srv.drain()
        assert srv.poll(a)["state"] == "done"


def test_nonfinite_request_fails_neighbours_unaffected(lib):
    from tarang_b200.serving import Server
    N = (32, 32, 32)
    good = fluid_fields(N, 11)
    bad = fluid_fields(N, 12)
    bad[1][1, 2, 3] = complex(float("nan"), 0.0)
    cfg = dict(N=N, nu=2e-3, dt=1e-3)
    with Server(hbm_budget=8e9, max_batch=4) as srv:
        rb = srv.submit(cfg, bad, 6)
        rg = srv.submit(cfg, good, 6)
        srv.drain()
        sb, sg = srv.poll(rb), srv.poll(rg)
        assert sb["state"] == "failed" and sb["error"] == L.TG_ERR_NONFINITE and sb["steps_done"] == 1
        assert sg["state"] == "done"
        want, _, _ = lone(cfg, good, 6)
        assert same_bits(srv.result(rg), want)


def test_bad_requests_rejected_at_submit(lib):
    from tarang_b200.serving import Server
    with Server(hbm_budget=1e9) as srv:
        with pytest.raises(L.TarangError) as e:
            srv.submit(dict(N=(32, 32, 30)), fluid_fields((32, 32, 30), 1), 3)   # N3/2 not a power of two
        assert e.value.code == L.TG_ERR_UNSUPPORTED
        with pytest.raises(L.TarangError) as e:
            srv.submit(dict(N=(32, 32, 32), dt=-1.0), fluid_fields((32, 32, 32), 1), 3)
        assert e.value.code == L.TG_ERR_ARG
        with pytest.raises(ValueError):
            srv.submit(dict(N=(32, 32, 32)), fluid_fields((32, 32, 32), 1)[:2], 3)


def test_forced_request_runs_in_its_own_context(lib):
    from tarang_b200.serving import Server
    N = (32, 32, 32)
    force = dict(inner=2.0, outer=3.0, eps=0.1)
    cfg = dict(N=N, nu=1e-3, dt=5e-4, force=force)
    f1, f2 = fluid_fields(N, 21), fluid_fields(N, 22)
    with Server(hbm_budget=8e9, max_batch=8) as srv:
        a = srv.submit(cfg, f1, 5)
        b = srv.submit(cfg, f2, 5)
        srv.pump()
        assert srv.stats()["n_batches"] == 2
        srv.drain()
        for rid, f in ((a, f1), (b, f2)):
            want, _, _ = lone(cfg, f, 5)
            assert same_bits(srv.result(rid), want)


def test_served_request_matches_oracle(lib):
    """10 FP64 steps of a served Taylor-Green request against the oracle (rel L2 <= 1e-12)."""
    from tarang_b200.serving import Server
    N = (32, 32, 32)
    V = ic.taylor_green(N)
    with Server(hbm_budget=8e9) as srv:
        ids = [srv.submit(dict(N=N, nu=0.01, dt=1e-3), V, 10)]
        ids.append(srv.submit(dict(N=N, nu=0.02, dt=1e-3), fluid_fields(N, 5), 10))
        srv.drain()
        got = srv.result(ids[0])
    ref = o.FluidSolver(N, KF, 0.01, 1e-3)
    Vw = V
    for _ in range(10):
        Vw, _ = ref.step(Vw)
    num = math.sqrt(sum(float(np.sum(np.abs(x - y) ** 2)) for x, y in zip(got, Vw)))
    den = math.sqrt(sum(float(np.sum(np.abs(y) ** 2)) for y in Vw))
    assert num / den < 1e-12


def test_zero_step_request_returns_stored_fields(lib):
    from tarang_b200.serving import Server
    from tarang_b200.solver import IncFluid
    N = (32, 32, 32)
    V = fluid_fields(N, 31)
    with Server(hbm_budget=8e9) as srv:
        a = srv.submit(dict(N=N), V, 0)
        b = srv.submit(dict(N=N, nu=5e-3), fluid_fields(N, 32), 3)
        srv.drain()
        st = srv.poll(a)
        assert st["state"] == "done" and st["steps_done"] == 0
        got = srv.result(a)
        srv.release(a)
        with pytest.raises(L.TarangError):
            srv.result(a)
        assert srv.poll(b)["steps_done"] == 3
    s = IncFluid(N)
    s.set_V(V)
    assert same_bits(got, s.get_V())


def test_idle_batch_evicted_for_new_shape(lib):
    """An idle batch stays resident for its shape and is released when a request of another
    shape needs its memory."""
    from tarang_b200.serving import Server, request_bytes
    a_cfg = dict(N=(32, 32, 32), nu=2e-3, dt=1e-3)
    b_cfg = dict(N=(16, 16, 32), nu=2e-3, dt=1e-3)
    budget = request_bytes(a_cfg, 1) + request_bytes(b_cfg, 1) // 2
    fa, fb = fluid_fields((32, 32, 32), 801), fluid_fields((16, 16, 32), 802)
    with Server(hbm_budget=budget, max_batch=4) as srv:
        a = srv.submit(a_cfg, fa, 4)
        srv.drain()
        s = srv.stats()
        assert s["n_batches"] == 1 and s["bytes_resident"] == request_bytes(a_cfg, 1)
        b = srv.submit(b_cfg, fb, 4)
        srv.drain()
        s = srv.stats()
        assert s["n_batches"] == 1 and s["bytes_resident"] == request_bytes(b_cfg, 1)
        assert s["bytes_peak"] <= budget
        for rid, cfg, f in ((a, a_cfg, fa), (b, b_cfg, fb)):
            assert srv.poll(rid)["state"] == "done"
            want, _, _ = lone(cfg, f, 4)
            assert same_bits(srv.result(rid), want)
