"""The batched / served engine (aed_server_*): parity with single solves, batch
independence, admission by HBM footprint, continuous batching (needs a B200)."""

from math import comb

import numpy as np
import pytest

import alps_b200 as ed
import oracle

pytestmark = pytest.mark.gpu


def j1j2(L, j2):
    out = []
    for i in range(L):
        out.append((i, (i + 1) % L, 1.0, 1.0))
        out.append((i, (i + 2) % L, float(j2), float(j2)))
    return out


def ladder(L, jl, jr):
    # anisotropic2d cell order: leg (x,y)->(x+1,y) type 0, rung (x,0)->(x,1) type 1; site = 2x + y
    out = []
    for x in range(L):
        for y in range(2):
            s = 2 * x + y
            out.append((s, 2 * ((x + 1) % L) + y, jl, jl))
            if y == 0:
                out.append((s, s + 1, jr, jr))
    return out


def reference(n, bonds, nev):
    ham = ed.Hamiltonian(n, n // 2, bonds)
    r = ham.solve(nev=nev, seed=3)
    ham.close()
    return r["evals"]


def mixed_requests(seed, count):
    rng = np.random.default_rng(seed)
    reqs = []
    for k in range(count):
        if rng.random() < 0.6:
            L = int(rng.choice([10, 12, 14, 16, 18]))
            reqs.append((L, j1j2(L, rng.uniform(0, 1)), int(rng.integers(1, 4)), int(rng.integers(0, 1 << 30))))
        else:
            L = int(rng.choice([5, 6, 7, 8]))
            reqs.append((2 * L, ladder(L, rng.uniform(0.5, 1.5), rng.uniform(0.5, 1.5)), int(rng.integers(1, 4)),
                         int(rng.integers(0, 1 << 30))))
    return reqs


@pytest.mark.parametrize("prec,tol", [(ed.FP32, 1e-9), (ed.FP64, 1e-11)])
def test_batch_matches_single_solves(prec, tol):
    reqs = mixed_requests(5124, 24)
    srv = ed.Server(precision=prec, max_slots=64, steps=8)
    tickets = [srv.submit(n, n // 2, b, nev=nev, seed=sd) for n, b, nev, sd in reqs]
    res = srv.run(tickets)
    for t, (n, b, nev, sd) in zip(tickets, reqs):
        r = res[t]
        ref = reference(n, b, nev)
        assert r["converged"]
        assert len(r["evals"]) == len(ref)
        rel = np.abs(r["evals"] - ref) / np.abs(ref)
        assert np.all(rel <= tol), (n, nev, rel)
        if prec == ed.FP32:
            assert r["iterations_low"] > 0
    srv.close()


@pytest.mark.parametrize("prec,tol", [(ed.FP32, 1e-9), (ed.FP64, 1e-11)])
def test_batch_matches_oracle(prec, tol):
    """The batched engine against the oracle directly (not through the single-instance CUDA path):
    each request's eigenvalues against the oracle's ietl-faithful Lanczos from the same start
    vector (lanczos.h:341-406, tmatrix.h:121-228) on its explicit matrix, and the ground state
    against a dense eigensolve where the sector is small."""
    reqs = mixed_requests(4242, 16)
    srv = ed.Server(precision=prec, max_slots=32, steps=8)
    tickets = [srv.submit(n, n // 2, b, nev=nev, seed=sd) for n, b, nev, sd in reqs]
    res = srv.run(tickets)
    for t, (n, b, nev, sd) in zip(tickets, reqs):
        M = oracle.Matrix(n, n // 2, [tuple(x) + (0.0,) for x in b])
        o = M.lanczos(nev=nev, seed=sd)
        r = res[t]
        assert r["converged"] and o["fail"] == 0
        assert len(r["evals"]) == len(o["evals"]), (n, nev, r["evals"], o["evals"])
        rel = np.abs(r["evals"] - o["evals"]) / np.abs(o["evals"])
        assert np.all(rel <= tol), (n, nev, rel)
        if M.D <= 1000:
            assert abs(r["evals"][0] - np.linalg.eigvalsh(M.dense())[0]) <= tol * abs(r["evals"][0])
    srv.close()


def test_batched_rayleigh_ritz_hand_over_bounds_hold():
    """Mixed batch: requests whose FP32 phase ends go through the batched Rayleigh-Ritz step first.  Most
    take its result (refined_by 'rayleigh_ritz', K FP64 applies); every value lies above the oracle's by at
    most its reported bound (the block Kato-Temple bound of the step) and within 1e-9; the others took the
    FP64 Lanczos refinement."""
    reqs = mixed_requests(99, 16)
    srv = ed.Server(precision=ed.FP32, max_slots=32, steps=8)
    tickets = [srv.submit(n, n // 2, b, nev=nev, seed=sd) for n, b, nev, sd in reqs]
    res = srv.run(tickets)
    kinds = [res[t]["refined_by"] for t in tickets]
    assert kinds.count("rayleigh_ritz") >= len(tickets) // 2, kinds
    assert set(kinds) <= {"rayleigh_ritz", "lanczos"}
    for t, (n, b, nev, sd) in zip(tickets, reqs):
        r = res[t]
        o = oracle.Matrix(n, n // 2, [tuple(x) + (0.0,) for x in b]).lanczos(nev=nev, seed=sd)
        assert len(r["evals"]) == len(o["evals"])
        assert np.all(np.abs(r["evals"] - o["evals"]) <= 1e-9 * np.abs(o["evals"]))
        if r["refined_by"] == "rayleigh_ritz":
            assert r["iterations"] <= 8  # the FP64 applies of the step
            assert np.all(r["evals"] - o["evals"] <= r["errors"] + 1e-12 * np.abs(o["evals"]))
    srv.close()


def test_batched_apply_candidates_give_the_same_results(monkeypatch):
    """The autotuner of the batched engine picks one of several FP32 apply kernels per sector-size bucket
    (rows per thread, CTAs per SM, hi blocks per pass); each adds every row's terms in the same order, so
    forcing any one of them (AED_BATCH_VARIANT) gives the same eigenvalues bit for bit, and the tuned
    server gives them too."""
    reqs = mixed_requests(31, 10)
    got = []
    for cand in [None, 0, 1, 2, 3, 4]:
        if cand is None:
            monkeypatch.delenv("AED_BATCH_VARIANT", raising=False)
        else:
            monkeypatch.setenv("AED_BATCH_VARIANT", str(cand))
        srv = ed.Server(precision=ed.FP32, max_slots=32, steps=4)
        ts = [srv.submit(n, n // 2, b, nev=nev, seed=sd) for n, b, nev, sd in reqs]
        res = srv.run(ts)
        got.append([res[t]["evals"].tolist() for t in ts])
        srv.close()
    for g in got[1:]:
        assert g == got[0]


@pytest.mark.parametrize("prec,tol", [(ed.FP32, 1e-9), (ed.FP64, 1e-11)])
def test_large_requests_run_in_single_instance_lanes(prec, tol):
    """Requests at or above lane_min_dim run as single-instance solves on their own handle, beside the
    batch: the mix finishes, lanes were in use, every result agrees with the single-instance solve of the
    same request (to the tolerance of the batched test), and a lane result is the same alone and in the mix."""
    reqs = mixed_requests(777, 14)
    srv = ed.Server(precision=prec, max_slots=32, steps=4, max_lanes=2, lane_min_dim=10000)
    ts = [srv.submit(n, n // 2, b, nev=nev, seed=sd) for n, b, nev, sd in reqs]
    seen_lanes = 0
    out = {}
    for _ in range(100000):
        if len(out) == len(ts):
            break
        srv.step()
        seen_lanes = max(seen_lanes, srv.stats()["lanes"])
        for t in ts:
            if t not in out:
                r = srv.poll(t)
                if r is not None:
                    out[t] = r
    assert len(out) == len(ts) and seen_lanes >= 1
    for t, (n, b, nev, sd) in zip(ts, reqs):
        ref = reference(n, b, nev)
        assert out[t]["converged"] and len(out[t]["evals"]) == len(ref)
        assert np.all(np.abs(out[t]["evals"] - ref) <= tol * np.abs(ref)), (n, out[t]["evals"], ref)
    big = [(t, q) for t, q in zip(ts, reqs) if comb(q[0], q[0] // 2) >= 10000]
    assert big
    t0, (n, b, nev, sd) = big[0]
    alone = ed.Server(precision=prec, max_slots=4, steps=4, max_lanes=1, lane_min_dim=10000)
    ta = alone.submit(n, n // 2, b, nev=nev, seed=sd)
    ra = alone.run([ta])[ta]
    alone.close()
    assert np.array_equal(ra["evals"], out[t0]["evals"])
    srv.close()


@pytest.mark.parametrize("prec", [ed.FP32, ed.FP64])
def test_result_is_the_same_alone_and_in_the_mix(prec):
    probe = (16, j1j2(16, 0.37), 2, 77)
    alone = ed.Server(precision=prec, max_slots=8, steps=4)
    t = alone.submit(16, 8, probe[1], nev=2, seed=77)
    r_alone = alone.run([t])[t]
    alone.close()
    srv = ed.Server(precision=prec, max_slots=32, steps=4)
    others = mixed_requests(99, 12)
    ts = [srv.submit(n, n // 2, b, nev=nev, seed=sd) for n, b, nev, sd in others[:6]]
    srv.step()  # the probe arrives while others are resident
    tp = srv.submit(16, 8, probe[1], nev=2, seed=77)
    srv.step()
    ts += [srv.submit(n, n // 2, b, nev=nev, seed=sd) for n, b, nev, sd in others[6:]]
    res = srv.run(ts + [tp])
    r_mix = res[tp]
    assert np.array_equal(r_mix["evals"], r_alone["evals"])
    assert r_mix["iterations"] == r_alone["iterations"]
    srv.close()


def test_admission_by_hbm_footprint_queues_and_refuses():
    rng = np.random.default_rng(7)
    reqs = [(18, j1j2(18, rng.uniform(0, 1)), 1, k) for k in range(10)]
    budget = 64 << 20  # an L=18 request holds ~30 MB: two resident at a time
    srv = ed.Server(precision=ed.FP32, max_slots=64, hbm_budget=budget)
    tickets = [srv.submit(n, n // 2, b, nev=nev, seed=sd) for n, b, nev, sd in reqs]
    srv.step()
    st = srv.stats()
    assert st["bytes_used"] <= budget
    assert st["queued"] > 0 and st["resident"] >= 1
    res = srv.run(tickets)
    assert len(res) == len(tickets)
    with pytest.raises(ed.AEDError) as e:
        srv.submit(24, 12, j1j2(24, 0.2), nev=1)
    assert e.value.code == ed.ERR_ADMISSION
    srv.close()


def test_cancel_and_continuous_batching():
    srv = ed.Server(precision=ed.FP32, max_slots=16, steps=2)
    a = srv.submit(18, 9, j1j2(18, 0.3), nev=1, seed=1)
    c = srv.submit(14, 7, j1j2(14, 0.6), nev=1, seed=2)
    srv.cancel(c)
    srv.step()
    b = srv.submit(12, 6, j1j2(12, 0.8), nev=1, seed=3)  # joins while a is resident
    overlap = False
    done = {}
    for _ in range(2000):
        srv.step()
        st = srv.stats()
        if st["resident"] >= 2:
            overlap = True
        for t in (a, b):
            if t not in done:
                r = srv.poll(t)
                if r is not None:
                    done[t] = r
        if len(done) == 2:
            break
    assert overlap and len(done) == 2
    with pytest.raises(ed.AEDError) as e:
        srv.poll(c)
    assert e.value.code == ed.ERR_CANCELLED
    assert done[b]["seconds"] > 0
    srv.close()


def test_reserved_pool_serves_requests():
    """A server that maps its budget into the memory pool at creation gives the same results."""
    reqs = mixed_requests(77, 6)
    srv = ed.Server(precision=ed.FP32, max_slots=16, steps=8, hbm_budget=1 << 30, reserve=-1)
    tickets = [srv.submit(n, n // 2, b, nev=nev, seed=sd) for n, b, nev, sd in reqs]
    res = srv.run(tickets)
    for t, (n, b, nev, sd) in zip(tickets, reqs):
        ref = reference(n, b, nev)
        assert np.all(np.abs(res[t]["evals"] - ref) / np.abs(ref) <= 1e-9)
    srv.close()
