"""The device-resident serving loop (sp_server_*): results against the
oracle's finite-difference tangent (micro/src/homogenize.c:59-94), the same
request alone and in a mix of concurrent requests, the replay driver, and
admission by HBM budget."""
import ctypes as C
import time

import numpy as np
import pytest

import madmax_b200 as mb
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def geoms():
    rng = np.random.default_rng(17)
    out = []
    for n in (3, 4, 5, 6, 4, 8):
        ratio = float(np.exp(rng.uniform(np.log(2), np.log(100))))
        out.append(mb.rve_desc(n, float(rng.uniform(0.1, 0.35)), (1e9, 1e9 * ratio),
                               (float(rng.uniform(0.2, 0.35)), float(rng.uniform(0.2, 0.35)))))
    return out


def oracle_fd(d, eps):
    m = O.cube_mesh(d.n[0])
    et = O.fiber_types(m, [1, 1], d.radius)
    Cm, s0 = O.fd_tangent(m, et, (d.E[0], d.E[1]), (d.nu[0], d.nu[1]), eps, rtol=1e-12,
                          lin_rtol=1e-13)
    return s0, Cm


@pytest.mark.parametrize("op", [mb.SP_OP_STENCIL, mb.SP_OP_ELL])
def test_serve_matches_oracle(op):
    G = geoms()
    s = mb.Server(G, op=op)
    s.start()
    rng = np.random.default_rng(1)
    reqs = [(int(rng.integers(0, len(G))), rng.normal(0, 1e-3, 6)) for _ in range(12)]
    tickets = [s.submit(g, e) for g, e in reqs]
    for tk, (g, e) in zip(tickets, reqs):
        st, tg, info = s.wait(tk)
        assert info.status == 0 and info.relres <= 1e-8
        s0, Cm = oracle_fd(G[g], e)
        assert np.abs(st - s0).max() <= 1e-8 * np.abs(s0).max()
        assert np.abs(tg - Cm).max() <= 1e-7 * np.abs(Cm).max()
    s.stop()
    s.close()


def test_same_result_alone_and_in_mix():
    G = geoms()
    e = np.array([1e-3, -5e-4, 2e-4, 3e-4, 0.0, -1e-4])
    a = mb.Server(G)
    a.start()
    st_alone, tg_alone, _ = a.wait(a.submit(3, e))
    a.stop()
    a.close()
    b = mb.Server(G)
    b.start()
    rng = np.random.default_rng(2)
    burst = [b.submit(int(rng.integers(0, len(G))), rng.normal(0, 1e-3, 6)) for _ in range(20)]
    mine = b.submit(3, e)
    burst += [b.submit(int(rng.integers(0, len(G))), rng.normal(0, 1e-3, 6)) for _ in range(20)]
    st_mix, tg_mix, info = b.wait(mine)
    for tk in burst:
        assert b.wait(tk)[2].status == 0
    b.stop()
    b.close()
    # warm starts differ between the two runs: equal within the solve tolerance
    assert np.abs(st_mix - st_alone).max() <= 2e-8 * np.abs(st_alone).max()
    assert np.abs(tg_mix - tg_alone).max() <= 2e-7 * np.abs(tg_alone).max()


def test_replay_poisson_latencies():
    G = geoms()
    s = mb.Server(G)
    rng = np.random.default_rng(3)
    n = 200
    t_arr = np.cumsum(rng.exponential(1.0 / 2000.0, size=n))
    geo = rng.integers(0, len(G), size=n)
    eps = rng.normal(0, 1e-3, size=(n, 6))
    td, st, tg, info = s.replay(geo, eps, t_arr, timeout=120)
    lat = td - t_arr
    assert (lat > 0).all()
    assert all(i.status == 0 for i in info)
    # spot-check a few against the oracle
    for i in (0, 57, 199):
        s0, Cm = oracle_fd(G[geo[i]], eps[i])
        assert np.abs(st[i] - s0).max() <= 1e-8 * np.abs(s0).max()
    s.stop()
    s.close()


def test_budget_refusal_and_bad_geometry():
    G = geoms()
    descs = (mb.sp_rve_desc * len(G))(*G)
    o = mb.server_opts(hbm_budget=1 << 20)
    h = mb._vp()
    assert mb.lib().sp_server_create(len(G), descs, C.byref(o), C.byref(h)) == mb.SP_ERR_BUDGET
    s = mb.Server(G)
    s.start()
    t = C.c_longlong()
    e = np.zeros(6)
    assert mb.lib().sp_server_submit(s.h, len(G), mb.ptr(e), C.byref(t)) == mb.SP_ERR_RANGE
    s.stop()
    s.close()


def test_repeated_and_zero_strain_requests_converge():
    """A warm start that already solves the request (the same strain again)
    stops at once, and a zero strain (zero right-hand side of the base load
    case) is answered with zero stress: the stopping rule is relative to the
    right-hand side, not to the warm start's residual."""
    G = geoms()
    s = mb.Server(G)
    s.start()
    e = np.array([2e-4, -1e-4, 3e-4, 0.0, 1e-4, -2e-4])
    st1, tg1, i1 = s.wait(s.submit(2, e))
    st2, tg2, i2 = s.wait(s.submit(2, e))
    z = np.zeros(6)
    st0, tg0, i0 = s.wait(s.submit(2, z))
    st0b, tg0b, i0b = s.wait(s.submit(2, z))
    s.stop()
    s.close()
    for i in (i1, i2, i0, i0b):
        assert i.status == 0 and i.relres <= 1e-8
    assert i2.inner_its < i1.inner_its
    assert np.abs(st2 - st1).max() <= 2e-8 * np.abs(st1).max()
    assert np.abs(st0).max() <= 1e-9 * np.abs(st1).max()
    assert np.abs(tg0 - tg1).max() <= 1e-7 * np.abs(tg1).max()
    assert np.abs(tg0b - tg1).max() <= 1e-7 * np.abs(tg1).max()


def test_warm_last_mode_solves_every_request():
    """SP_WARM_LAST: each request starts from the geometry's last solution
    of each load case (no prediction), runs CG to 1e-8, and keeps its
    solution as the next start; results match the oracle."""
    G = geoms()
    s = mb.Server(G, warm_start=mb.SP_WARM_LAST)
    s.start()
    rng = np.random.default_rng(8)
    reqs = [(g, rng.normal(0, 1e-3, 6)) for g in (2, 5, 2, 5, 2)]
    res = [s.wait(s.submit(g, e)) for g, e in reqs]
    s.stop()
    s.close()
    for (st, tg, info), (g, e) in zip(res, reqs):
        assert info.status == 0 and info.relres <= 1e-8 and info.outer_its > 0
        s0, Cm = oracle_fd(G[g], e)
        assert np.abs(st - s0).max() <= 1e-8 * np.abs(s0).max()
        assert np.abs(tg - Cm).max() <= 1e-7 * np.abs(Cm).max()
    bad = mb.server_opts(warm_start=7)
    descs = (mb.sp_rve_desc * len(G))(*G)
    h = mb._vp()
    assert mb.lib().sp_server_create(len(G), descs, C.byref(bad), C.byref(h)) == mb.SP_ERR_ARG


def test_idle_loop_returns_and_is_relaunched():
    """Every device wait of the serving loop is bounded: with a small
    idle_spin_limit the loop returns by itself once its queue stays empty
    (the host sees its stream idle), and the next submit relaunches it; the
    answers before and after match the oracle."""
    G = geoms()
    s = mb.Server(G, idle_spin_limit=1000)
    s.start()
    e1 = np.array([3e-4, -1e-4, 2e-4, 0.0, 1e-4, -2e-4])
    st1, tg1, i1 = s.wait(s.submit(1, e1))
    deadline = time.time() + 20.0
    on, n1, _ = s.status()
    while on and time.time() < deadline:
        time.sleep(0.01)
        on, n1, _ = s.status()
    assert not on and n1 == 1
    e2 = np.array([-2e-4, 4e-4, 1e-4, 2e-4, 0.0, 1e-4])
    st2, tg2, i2 = s.wait(s.submit(3, e2))
    _, n2, sub = s.status()
    s.stop()
    s.close()
    assert n2 == 2 and sub == 2
    for st, tg, info, g, e in ((st1, tg1, i1, 1, e1), (st2, tg2, i2, 3, e2)):
        assert info.status == 0 and info.relres <= 1e-8
        s0, Cm = oracle_fd(G[g], e)
        assert np.abs(st - s0).max() <= 1e-8 * np.abs(s0).max()
        assert np.abs(tg - Cm).max() <= 1e-7 * np.abs(Cm).max()


# --------------------------------------- message_t coupling (micro side) ---

def fake_transport(inbox):
    """In-memory stand-in for the MPI transport: recv pops the next queued
    message, send records the reply."""
    sent = []

    def recv(msg, ctx):
        if not inbox:
            return 1
        C.memmove(msg, C.byref(inbox.pop(0)), C.sizeof(mb.sp_message))
        return 0

    def send(msg, ctx):
        m = mb.sp_message()
        C.memmove(C.byref(m), msg, C.sizeof(mb.sp_message))
        sent.append(m)
        return 0

    return mb.MESSAGE_RECV(recv), mb.MESSAGE_SEND(send), sent


def message(action, strain=None):
    m = mb.sp_message()
    m.action, m.num_voigt = action, 6
    if strain is not None:
        m.strain_mac[:] = list(strain)
    return m


@pytest.mark.parametrize("mode", [mb.SP_MICRO_SOLVE, mb.SP_MICRO_LINEAR])
def test_micro_message_loop_matches_oracle(mode):
    """The request loop of micro/src/main.c:114-153 over message_t: stress,
    tangent and density requests answered from the serving loop, END ends
    the loop unanswered; results against the oracle's FD tangent."""
    G = geoms()
    s = mb.Server(G)
    s.start()
    h = mb._vp()
    mb.check(mb.lib().sp_micro_create(s.h, 4, mode, 1e7, C.byref(h)), "sp_micro_create")
    e = np.array([4e-4, -2e-4, 1e-4, 3e-4, -1e-4, 2e-4])
    inbox = [message(mb.SP_ACTION_MICRO_CALC_STRESS, e), message(mb.SP_ACTION_MICRO_CALC_C_TANGENT, e),
             message(mb.SP_ACTION_MICRO_CALC_RHO), message(mb.SP_ACTION_MICRO_END)]
    recv, send, sent = fake_transport(inbox)
    n = C.c_longlong()
    mb.check(mb.lib().sp_micro_serve(h, recv, send, None, C.byref(n)), "sp_micro_serve")
    assert n.value == 4 and len(sent) == 3 and not inbox
    assert [m.action for m in sent] == [1, 2, 3]
    stress = np.array(sent[0].stress_ave[:])
    tangent = np.array(sent[1].c_tangent_ave[:]).reshape(6, 6)
    assert sent[2].rho == 1e7
    s0, Cm = oracle_fd(G[4], e)
    _, C0 = oracle_fd(G[4], np.zeros(6))
    if mode == mb.SP_MICRO_SOLVE:
        assert np.abs(stress - s0).max() <= 1e-8 * np.abs(s0).max()
        assert np.abs(tangent - Cm).max() <= 1e-7 * np.abs(Cm).max()
    else:
        # the reference's linear path: C from the FD tangent around zero, sigma = C eps
        assert np.abs(tangent - C0).max() <= 1e-7 * np.abs(C0).max()
        assert np.abs(stress - C0 @ e).max() <= 1e-7 * np.abs(C0 @ e).max()
    req = C.c_longlong()
    mb.lib().sp_micro_requests(h, C.byref(req))
    assert req.value == (2 if mode == mb.SP_MICRO_SOLVE else 1)
    bad = message(9)
    assert mb.lib().sp_micro_handle(h, C.byref(bad)) == mb.SP_ERR_ARG
    bad = message(mb.SP_ACTION_MICRO_CALC_STRESS, e)
    bad.num_voigt = 3
    assert mb.lib().sp_micro_handle(h, C.byref(bad)) == mb.SP_ERR_ARG
    mb.lib().sp_micro_destroy(h)
    s.stop()
    s.close()
