"""GPU tests of the serving engine (fa_server_*): continuous batching.

A session's results must not depend on what else the server is doing: every
request's observations and every instance's final state equal the oracle
stepping that session alone, whether the session is served alone, mixed with
other sessions submitted from several threads, or by the plain per-frame
form.  Admission under a state budget waits in FIFO order.
"""
import threading

import numpy as np
import pytest

import oracle
from fa_pkg import carts, fa
from test_gpu_parity import assert_states_equal

pytestmark = pytest.mark.gpu

BLOCK_BYTES = 67 * 256 * 4      # one state block of the server (FA_ROWS x 256 words)


@pytest.fixture(scope="module", autouse=True)
def need_gpu():
    if fa.device_count() < 1:
        pytest.skip("no CUDA device")


@pytest.fixture(scope="module")
def mixed():
    return carts.mixed_carts()


# Sessions: (cart index, [(n, k), ...]).  Sizes grow and shrink (instances
# beyond a request's n keep their state), cross 256-instance blocks and
# 128-instance units, and frame counts differ between requests.
SCRIPT = [
    (0, [(40, 3), (300, 2), (100, 5), (520, 1)]),
    (1, [(257, 4), (16, 1), (257, 2)]),
    (2, [(128, 2), (129, 3), (64, 6)]),
    (3, [(33, 5), (300, 1)]),
    (0, [(700, 2), (1, 3)]),
    (1, [(90, 7)]),
]


def script_actions(si, ri, n, k):
    return carts.actions(seed=1000 + 31 * si + ri, n=n, frames=k)


def oracle_session(rom, reqs, si):
    """Observations per request and the final states of one session, stepped alone."""
    snap = oracle.reset_state(rom)
    states = np.zeros(0, dtype=oracle.STATE_DTYPE)
    obs = []
    for ri, (n, k) in enumerate(reqs):
        if n > len(states):
            states = np.concatenate([states, np.array([snap] * (n - len(states)), dtype=oracle.STATE_DTYPE)])
        sub = np.ascontiguousarray(states[:n])
        o, _ = oracle.run_batch(rom, sub, script_actions(si, ri, n, k), k)
        states[:n] = sub
        obs.append(o)
    return obs, states


@pytest.fixture(scope="module")
def expected(mixed):
    return [oracle_session(mixed[c].rom, reqs, si) for si, (c, reqs) in enumerate(SCRIPT)]


def run_mixed(srv, threads=True):
    """Every session's requests from its own thread (closed loop), all at once."""
    sids = [srv.open(c) for c, _ in SCRIPT]
    got = [[None] * len(reqs) for _, reqs in SCRIPT]
    errors = []

    def client(si):
        try:
            _, reqs = SCRIPT[si]
            for ri, (n, k) in enumerate(reqs):
                got[si][ri], _ = srv.step(sids[si], script_actions(si, ri, n, k), n, k)
        except Exception as e:          # surfaced below
            errors.append(e)

    if threads:
        ts = [threading.Thread(target=client, args=(si,)) for si in range(len(SCRIPT))]
        for t in ts:
            t.start()
        for t in ts:
            t.join()
    else:
        # Submit everything up front (each session's requests queue behind
        # one another), then wait.
        tickets = [[srv.submit(sids[si], script_actions(si, ri, n, k), n, k) for ri, (n, k) in enumerate(reqs)]
                   for si, (_, reqs) in enumerate(SCRIPT)]
        for si, ts in enumerate(tickets):
            for ri, t in enumerate(ts):
                got[si][ri], _ = srv.wait(t)
    assert not errors, errors
    states = [srv.states(s) for s in sids]
    return got, states, sids


def check(got, states, expected, what):
    for si, (obs_exp, st_exp) in enumerate(expected):
        for ri, o in enumerate(obs_exp):
            assert np.array_equal(got[si][ri], o), f"{what}: session {si} request {ri}"
        assert_states_equal(states[si], st_exp, f"{what}: session {si}")


@pytest.mark.parametrize("threads", [True, False])
def test_mixed_sessions_match_oracle(mixed, expected, threads):
    with fa.AtariServer([c.rom for c in mixed]) as srv:
        got, states, _ = run_mixed(srv, threads)
        st = srv.stats()
    check(got, states, expected, "batched")
    n_req = sum(len(r) for _, r in SCRIPT)
    assert st["requests_done"] == n_req and st["requests_failed"] == 0
    assert st["instance_frames"] == sum(n * k for _, r in SCRIPT for n, k in r)
    assert st["guest_instructions"] > 0
    # how requests group into batches depends on timing; each is dispatched once
    assert st["dispatched_requests"] == n_req and 1 <= st["dispatches"] <= n_req


@pytest.mark.parametrize("block", [128, 256])     # the default is 512
def test_batched_cta_sizes_match_oracle(mixed, expected, block):
    with fa.AtariServer([c.rom for c in mixed], block=block, max_inflight=3) as srv:
        got, states, _ = run_mixed(srv, threads=False)
    check(got, states, expected, f"batched/{block}")


def test_each_session_alone_equals_in_the_mix(mixed, expected):
    # Alone: one session at a time on a fresh server, one request at a time.
    alone_obs, alone_states = [], []
    with fa.AtariServer([c.rom for c in mixed]) as srv:
        for si, (c, reqs) in enumerate(SCRIPT):
            sid = srv.open(c)
            obs = [srv.step(sid, script_actions(si, ri, n, k), n, k)[0] for ri, (n, k) in enumerate(reqs)]
            alone_obs.append(obs)
            alone_states.append(srv.states(sid))
            srv.close_session(sid)
    with fa.AtariServer([c.rom for c in mixed]) as srv:
        mix_obs, mix_states, _ = run_mixed(srv, threads=True)
    for si in range(len(SCRIPT)):
        for ri in range(len(SCRIPT[si][1])):
            assert np.array_equal(alone_obs[si][ri], mix_obs[si][ri]), f"session {si} request {ri}"
        assert_states_equal(mix_states[si], alone_states[si], f"session {si}")
    check(alone_obs, alone_states, expected, "alone")


@pytest.mark.parametrize("block", [128, 256])
def test_plain_mode_matches_oracle(mixed, expected, block):
    with fa.AtariServer([c.rom for c in mixed], mode="plain", block=block) as srv:
        got, states, _ = run_mixed(srv, threads=False)
        st = srv.stats()
    check(got, states, expected, f"plain/{block}")
    # one launch per frame per cart of each static batch
    assert st["launches"] >= max(k for _, r in SCRIPT for _, k in r)


def test_admission_waits_fifo_under_budget(mixed):
    rom = mixed[0].rom
    snap = oracle.reset_state(rom)
    with fa.AtariServer([rom], state_budget_bytes=3 * BLOCK_BYTES) as srv:
        a, b, c = srv.open(0), srv.open(0), srv.open(0)
        acts_a = carts.actions(seed=5, n=512, frames=2)
        obs_a, info = srv.step(a, acts_a, 512, 2)                 # 2 of 3 blocks
        assert info["waited_admission"] == 0
        tb = srv.submit(b, carts.actions(seed=6, n=300, frames=2), 300, 2)   # needs 2: waits
        tc = srv.submit(c, carts.actions(seed=7, n=10, frames=3), 10, 3)     # needs 1, but FIFO: waits
        for t in (tb, tc):
            with pytest.raises(fa.FaError) as ei:
                srv.wait(t, timeout_ms=300)
            assert ei.value.code == fa.FA_ERR_TIMEOUT
        st = srv.stats()
        assert st["admission_waits"] == 2
        assert st["state_bytes_in_use"] == 2 * BLOCK_BYTES
        # A request larger than the whole budget can never be admitted.
        with pytest.raises(fa.FaError) as ei:
            srv.submit(c, np.zeros(1025 * 1, np.uint8), 1025, 1)
        assert ei.value.code == fa.FA_ERR_CAPACITY
        srv.close_session(a)                                      # frees 2 blocks
        obs_b, ib = srv.wait(tb)
        obs_c, ic = srv.wait(tc)
        assert ib["waited_admission"] == 1 and ic["waited_admission"] == 1
        assert srv.stats()["state_bytes_in_use"] == 3 * BLOCK_BYTES
    for n, k, seed, got in ((512, 2, 5, obs_a), (300, 2, 6, obs_b), (10, 3, 7, obs_c)):
        st = np.array([snap] * n, dtype=oracle.STATE_DTYPE)
        o, _ = oracle.run_batch(rom, st, carts.actions(seed=seed, n=n, frames=k), k)
        assert np.array_equal(got, o), f"n={n}"


def test_closed_session_runs_its_queue_then_frees(mixed):
    rom = mixed[1].rom
    with fa.AtariServer([rom]) as srv:
        s = srv.open(0)
        t1 = srv.submit(s, carts.actions(seed=8, n=200, frames=2), 200, 2)
        t2 = srv.submit(s, carts.actions(seed=9, n=200, frames=2), 200, 2)
        srv.close_session(s)
        o1, _ = srv.wait(t1)
        o2, _ = srv.wait(t2)
        assert srv.stats()["state_bytes_in_use"] == 0
        with pytest.raises(fa.FaError):
            srv.submit(s, np.zeros(4, np.uint8), 4, 1)
    st = np.array([oracle.reset_state(rom)] * 200, dtype=oracle.STATE_DTYPE)
    e1, _ = oracle.run_batch(rom, st, carts.actions(seed=8, n=200, frames=2), 2)
    e2, _ = oracle.run_batch(rom, st, carts.actions(seed=9, n=200, frames=2), 2)
    assert np.array_equal(o1, e1) and np.array_equal(o2, e2)


def test_loadgen_trace_same_work_in_both_modes(mixed):
    roms = [c.rom for c in mixed]
    kw = dict(requests=120, offered_frames_per_s=0.0, clients=8, seed=3, batch_median=64, batch_max=2048)
    with fa.AtariServer(roms) as srv:
        rb, lat_b = srv.loadgen(**kw)
        stb = srv.stats()
    with fa.AtariServer(roms, mode="plain") as srv:
        rp, lat_p = srv.loadgen(**kw)
    assert rb["errors"] == 0 and rp["errors"] == 0
    assert rb["requests"] == rp["requests"] == 120
    assert rb["instance_frames"] == rp["instance_frames"] == stb["instance_frames"]
    for rec, res in ((lat_b, rb), (lat_p, rp)):
        assert (rec["latency_ms"] > 0).all() and (rec["service_ms"] > 0).all()
        # the parts of every request's latency add up to it
        parts = rec["session_wait_ms"] + rec["dispatch_ms"] + rec["service_ms"]
        assert np.allclose(parts, rec["latency_ms"], rtol=0, atol=1e-6)
        assert (rec["session_wait_ms"] >= 0).all() and (rec["dispatch_ms"] >= -1e-9).all()
        assert float((rec["n"].astype(np.float64) * rec["k"]).sum()) == res["instance_frames"]
        assert set(np.unique(rec["cart"])) <= set(range(len(roms)))
    assert rb["p50_ms"] <= rb["p99_ms"] <= rb["max_ms"]
    assert stb["sessions_open"] == 0 and stb["state_bytes_in_use"] == 0
