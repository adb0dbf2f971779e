"""The continuous-batching request server (fmmb_server): requests of different sizes, point
distributions and tolerances submitted together run concurrently on several streams; each
result must be bitwise the same as the same request run alone, and within its tolerance of FP64
direct sums (relative L2 of the potential at sampled sources: 3·tol for tol ≥ 1e-6; 1e-8 for
tol = 1e-9, where p = 20 — the highest order provided — reaches ≈ 3e-9)."""
import numpy as np
import pytest

from helpers import rel_l2

pytestmark = pytest.mark.gpu


def _requests(seed, count, nmin=1000, nmax=60000):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = int(np.exp(rng.uniform(np.log(nmin), np.log(nmax))))
        if rng.random() < 0.5:
            pts = rng.random((n, 3))
        else:
            c = 0.1 + 0.8 * rng.random((4, 3))
            pts = np.clip(c[np.arange(n) % 4] + 0.02 * rng.standard_normal((n, 3)), 0.0, 1.0)
        tau = rng.standard_normal(n)
        tol = (1e-3, 1e-6, 1e-9)[i % 3]
        out.append((pts, tau, tol))
    return out


def test_server_mix_equals_alone_and_meets_tolerance(fmmb, oracle):
    reqs = _requests(5, 9)
    srv = fmmb.Server(0, slots=4)
    tickets = [srv.submit(p, t, tol=tol) for p, t, tol in reqs]          # all in flight together
    mixed = [srv.wait(k) for k in tickets]
    alone = []
    for p, t, tol in reqs:                                              # one at a time
        alone.append(srv.wait(srv.submit(p, t, tol=tol)))
    srv.close()
    slots = {info["slot"] for _, _, info in mixed}
    assert len(slots) > 1                                               # the mix ran on several streams
    rng = np.random.default_rng(0)
    for (pts, tau, tol), (u, g, info), (ua, ga, _) in zip(reqs, mixed, alone):
        assert np.array_equal(u, ua) and np.array_equal(g, ga), info
        assert info["precision"] == ("fp64" if tol < 1e-8 else "mixed")
        sel = np.sort(rng.choice(len(pts), min(300, len(pts)), replace=False))
        du, _ = oracle.direct_sample(pts, tau, sel)
        err = rel_l2(u[sel], du)
        assert err < (1e-8 if tol < 1e-8 else 3 * tol), (len(pts), tol, info["p"], err)
        assert info["latency_s"] >= info["run_s"] > 0


def test_server_budget_admits_in_order(fmmb):
    reqs = _requests(6, 5, 2000, 20000)
    srv = fmmb.Server(0, slots=3, hbm_budget=1)                         # every request alone on the device
    tickets = [srv.submit(p, t, tol=1e-6) for p, t, _ in reqs]
    infos = [srv.wait(k)[2] for k in tickets]
    srv.close()
    # with no room for two requests at once, each starts after the previous one ends
    starts = [i["queued_s"] for i in infos]
    assert all(i["status"] == 0 for i in infos)
    assert starts == sorted(starts)


def test_server_errors(fmmb):
    srv = fmmb.Server(0, slots=2)
    with pytest.raises(fmmb.ArgumentError):
        srv.submit(np.zeros((0, 3)), np.zeros(0))
    bad = np.random.default_rng(1).random((500, 3))
    bad[7, 1] = np.nan
    k = srv.submit(bad, np.ones(500), tol=1e-3)
    with pytest.raises(fmmb.ArgumentError, match="finite"):
        srv.wait(k)
    good = np.random.default_rng(2).random((3000, 3))
    u, g, info = srv.wait(srv.submit(good, np.ones(3000), tol=1e-3))    # the server keeps serving
    assert info["status"] == 0 and np.all(np.isfinite(u))
    srv.close()


def test_server_stokes_requests_mixed_with_laplace(fmmb):
    """Stokeslet requests (the batched Stokes workload: jittered unit-sphere points, N(0,1)³
    forces) submitted among Laplace requests: each velocity field is bitwise the same as the
    request alone, and within 3·tol of FP64 direct Stokeslet sums (p from the Stokes table)."""
    from helpers import sphere_points, stokes_direct
    rng = np.random.default_rng(9)
    stokes = []
    for i, tol in enumerate((1e-3, 1e-5, 1e-6)):
        n = int(rng.integers(20000, 60000))
        stokes.append((sphere_points(rng, n), rng.standard_normal((n, 3)), tol))
    lap = _requests(10, 3)
    srv = fmmb.Server(0, slots=4)
    tickets = []
    for (x, f, tol), (px, pt, ptol) in zip(stokes, lap):
        tickets.append(("s", srv.submit_stokes(x, f, tol=tol, ppl=200)))
        tickets.append(("l", srv.submit(px, pt, tol=ptol)))
    mixed = [srv.wait(k) for _, k in tickets]
    alone = [srv.wait(srv.submit_stokes(x, f, tol=tol, ppl=200)) for x, f, tol in stokes]
    srv.close()
    res = [m for (kind, _), m in zip(tickets, mixed) if kind == "s"]
    for (x, f, tol), (v, g, info), (va, _, _) in zip(stokes, res, alone):
        assert g is None and info["precision"] == "fp64" and info["status"] == 0
        assert np.array_equal(v, va), info
        sel = np.sort(rng.choice(len(x), 200, replace=False))
        err = rel_l2(v[sel], stokes_direct(x, f, sel))
        assert err < 3 * tol, (len(x), tol, info["p"], err)


def test_server_yukawa_requests(fmmb):
    """Yukawa3D(κ = 5) requests among Laplace ones (the serving workload's other half): the path
    chosen by the tolerance (FP64 below 1e-8 and above p = 11, else the tensor-core M2L), each
    result bitwise the same alone, within 3·tol of FP64 direct sums."""
    from helpers import yukawa_direct
    reqs = _requests(12, 6, 2000, 40000)
    srv = fmmb.Server(0, slots=4)
    tickets = [srv.submit(p, t, tol=tol, kappa=5.0 if i % 2 == 0 else None) for i, (p, t, tol) in enumerate(reqs)]
    mixed = [srv.wait(k) for k in tickets]
    alone = [srv.wait(srv.submit(p, t, tol=tol, kappa=5.0)) for i, (p, t, tol) in enumerate(reqs) if i % 2 == 0]
    srv.close()
    rng = np.random.default_rng(1)
    for (pts, tau, tol), (u, g, info), (ua, ga, _) in zip(reqs[::2], mixed[::2], alone):
        assert info["precision"] == ("fp64" if tol < 1e-8 or info["p"] > 11 else "mixed") and info["status"] == 0
        assert np.array_equal(u, ua) and np.array_equal(g, ga)
        sel = np.sort(rng.choice(len(pts), 300, replace=False))
        du = np.zeros(len(sel))
        for k, i in enumerate(sel):                      # self excluded
            m = np.ones(len(pts), bool)
            m[i] = False
            du[k] = yukawa_direct(pts[m], tau[m], pts[i:i + 1], 5.0)[0]
        err = rel_l2(u[sel], du)
        assert err < (1e-8 if tol < 1e-8 else 3 * tol), (len(pts), tol, info["p"], err)
