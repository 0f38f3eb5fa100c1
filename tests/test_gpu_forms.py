"""The three forms beside the plain method, on the GPU through the C ABI:

* precision: FP32 reconstruction/flux/divergence with a compensated hi/lo
  FP32 conserved state, against the FP64 path (itself pinned to the oracle);
* batching: many uneven grids in one persistent launch per stage -- each
  instance's result equals the same grid advanced alone;
* serving: a request stream through the continuous-batching loop -- every
  request finishes, and its result is the one it gets alone.
"""
from __future__ import annotations

import numpy as np
import pytest

import fvstuff_b200 as F
from cases import kh, prim_to_cons, rel_linf, riemann4, smooth, vortex

pytestmark = pytest.mark.gpu


def rel_l1(a, b):
    return float(np.sum(np.abs(a - b)) / np.sum(np.abs(b)))


def _run(prec, w, steps, **kw):
    s = F.Solver(w.shape[-1], precision=prec, **kw)
    s.set_state(w, interior=True)
    s.step(steps)
    st = s.sync()
    assert st.status == 0 and st.steps == steps
    return s, s.get_state(layout="cons", interior=True), st


def test_f32c_vortex_against_f64():
    """Moving isentropic vortex, periodic [-5,5]^2 at 128^2, 300 steps at CFL
    0.5: density within 1e-6 relative L1 of the FP64 run."""
    n, steps = 128, 300
    w = vortex(n)
    kw = dict(bc="periodic", x0=-5, y0=-5, length=10.0, cfl=0.5)
    _, c64, s64 = _run("f64", w, steps, **kw)
    _, c32, s32 = _run("f32c", w, steps, **kw)
    e_rho = rel_l1(c32[0], c64[0])
    e_inf = rel_linf(c32, c64)
    print("f32c vs f64 vortex 128^2 x %d: rel L1(rho) %.3e, rel Linf(cons) %.3e, t %.9f / %.9f"
          % (steps, e_rho, e_inf, s32.t, s64.t))
    assert e_rho <= 1e-6
    assert abs(s32.t - s64.t) <= 1e-6 * s64.t


def test_f32c_kh_short_against_f64():
    n, steps = 256, 100
    w = kh(n)
    _, c64, _ = _run("f64", w, steps, bc="periodic", cfl=0.5)
    _, c32, _ = _run("f32c", w, steps, bc="periodic", cfl=0.5)
    e = [rel_l1(c32[q], c64[q]) for q in range(4)]
    print("f32c vs f64 KH 256^2 x %d: rel L1 rho %.2e rhou %.2e rhov %.2e E %.2e" % (steps, *e))
    assert e[0] <= 1e-6


@pytest.mark.parametrize("tile", [0, 1, 2, 3, 4, 5, 6])
def test_f32c_tile_variants_against_f64(tile):
    """Every tile variant of the compensated kernel, on a ragged grid with
    reflecting walls (ghost images with negated momenta on all four sides)."""
    n, steps = 77, 40
    w = vortex(n)
    kw = dict(bc="reflect", x0=-5, y0=-5, length=10.0, cfl=0.5)
    _, c64, _ = _run("f64", w, steps, **kw)
    _, c32, _ = _run("f32c", w, steps, tile=tile, **kw)
    assert rel_l1(c32[0], c64[0]) <= 1e-6


def test_f32c_hilo_is_normalised_and_conservative():
    n = 64
    s = F.Solver(n, precision="f32c", bc="periodic")
    s.set_state(smooth(n, seed=3), interior=True)
    a = s.stats().sums
    s.step(50)
    b = s.stats().sums
    hi, lo = s.get_state_hilo()
    # |lo| <= ulp(hi)/2: the pair is a normalised double-float
    assert np.all(np.abs(lo) <= np.spacing(np.abs(hi)) * 0.5 + 1e-45)
    drift = [abs(b[q] - a[q]) / max(abs(a[q]), 1.0) for q in range(4)]
    print("f32c conserved-sum drift after 50 steps:", drift)
    assert max(drift) <= 1e-7


def test_f32c_graph_and_direct_agree():
    n = 48
    w = riemann4(n, seed=2)
    a = F.Solver(n, precision="f32c", bc="transmissive")
    b = F.Solver(n, precision="f32c", bc="transmissive")
    b.set_graph(False)
    for s in (a, b):
        s.set_state(w, interior=True)
        s.step(9)   # odd: exercises the graph pair plus one direct step
    assert np.array_equal(a.get_state(interior=True), b.get_state(interior=True))
    a.advance(0.05)
    b.advance(0.05)
    assert np.array_equal(a.get_state(interior=True), b.get_state(interior=True))


# --- batched form -------------------------------------------------------------

def _desc(n, seed, t_end):
    c = F.case_params("riemann4", 0.0, 0.0, 1.0, seed=seed)
    return F.Batch.desc(n, c, t_end, bc="transmissive", cfl=0.5), c


@pytest.mark.parametrize("prec", ["f32c", "f64"])
def test_batch_instances_match_alone(prec):
    sizes = [64, 96, 33, 128, 50, 160]
    b = F.Batch(precision=prec)
    ids, cases = [], []
    for k, n in enumerate(sizes):
        d, c = _desc(n, 100 + k, 0.05 + 0.01 * k)
        ids.append(b.add(d))
        cases.append((n, c, d.t_end))
    done = set()
    for _ in range(400):
        b.run(8)
        done.update(b.poll())
        if len(done) == len(sizes):
            break
    assert done == set(ids)
    for iid, (n, c, t_end) in zip(ids, cases):
        st = b.stats(iid)
        assert st.status == 0 and st.t == pytest.approx(t_end, rel=0, abs=1e-12)
        got = b.get_state(iid, n)
        s = F.Solver(n, precision=prec, bc="transmissive", cfl=0.5)
        s.init_case(c)
        s.advance(t_end)
        alone = s.get_state(interior=True)
        assert s.sync().steps == st.steps
        assert np.array_equal(got, alone), (iid, n, np.max(np.abs(got - alone)))
    for iid in ids:
        b.remove(iid)
    assert b.bytes_in_use() == 0


def test_batch_row_pair_variant_matches_alone():
    """The FP32c row-pair kernel (tile variant 6, used only when asked for)
    in a batch of ragged grids, bit for bit against each grid run alone with
    the same variant, and against variant 5 alone (the two kernels evaluate
    the same operations in the same order)."""
    sizes = [64, 33, 96, 50]
    b = F.Batch(precision="f32c", tile=6)
    ids, cases = [], []
    for k, n in enumerate(sizes):
        d, c = _desc(n, 200 + k, 0.04)
        ids.append(b.add(d))
        cases.append((n, c, d.t_end))
    done = set()
    for _ in range(400):
        b.run(8)
        done.update(b.poll())
        if len(done) == len(sizes):
            break
    assert done == set(ids)
    for iid, (n, c, t_end) in zip(ids, cases):
        st = b.stats(iid)
        assert st.status == 0
        got = b.get_state(iid, n)
        for tile in (6, 5):
            s = F.Solver(n, precision="f32c", bc="transmissive", cfl=0.5, tile=tile)
            s.init_case(c)
            s.advance(t_end)
            assert s.sync().steps == st.steps
            assert np.array_equal(got, s.get_state(interior=True)), (iid, n, tile)


def test_batch_join_midway_and_budget():
    b = F.Batch(precision="f32c", hbm_budget=F.Batch(precision="f32c").instance_bytes(64) * 2)
    d1, _ = _desc(64, 1, 0.04)
    d2, c2 = _desc(64, 2, 0.03)
    d3, _ = _desc(64, 3, 0.03)
    i1 = b.add(d1)
    b.run(3)
    i2 = b.add(d2)  # joins while i1 is mid-run
    with pytest.raises(F.FvbError) as e:
        b.add(d3)
    assert e.value.status == F._lib.ERR_NOMEM
    done = set()
    for _ in range(200):
        b.run(4)
        done.update(b.poll())
        if done == {i1, i2}:
            break
    assert done == {i1, i2}
    s = F.Solver(64, precision="f32c", bc="transmissive", cfl=0.5)
    s.init_case(c2)
    s.advance(0.03)
    assert np.array_equal(b.get_state(i2, 64), s.get_state(interior=True))
    b.remove(i1)
    i3 = b.add(d3)  # fits once i1's memory is released
    assert i3 >= 0


@pytest.mark.parametrize("prec", ["f32c", "f64"])
def test_batch_bad_instances_stay_isolated(prec):
    """instances whose initial state is not a state -- NaN density,
    negative density and pressure -- run as the reference's scheme runs them
    (its floors turn NaN and negative rho, p into 1e-14, its sound-speed
    clamp a NaN c^2 into 1e-14; a non-positive wave speed stops the
    instance); whatever they do, the good instances of the same batch finish
    exactly as they do alone"""
    b = F.Batch(precision=prec)
    good = []
    for k, n in enumerate((48, 64, 40)):
        d, c = _desc(n, 300 + k, 0.03)
        good.append((b.add(d), n, c))
    bad = []
    for n, params in ((56, dict(rho=float("nan"))), (32, dict(rho=-1.0, p=-1.0))):
        c = F.case_params("uniform", 0.0, 0.0, 1.0, **params)
        bad.append(b.add(F.Batch.desc(n, c, 0.03, bc="transmissive", cfl=0.5)))
    done = set()
    for _ in range(400):
        b.run(8)
        done.update(b.poll())
        if len(done) == 5:
            break
    assert len(done) == 5
    for iid in bad:
        assert b.stats(iid).status in (0, F._lib.ERR_BLOWUP, F._lib.ERR_DT_UNDERFLOW)
    for iid, n, c in good:
        st = b.stats(iid)
        assert st.status == 0 and st.t == pytest.approx(0.03, rel=0, abs=1e-12)
        s = F.Solver(n, precision=prec, bc="transmissive", cfl=0.5)
        s.init_case(c)
        s.advance(0.03)
        assert np.array_equal(b.get_state(iid, n), s.get_state(interior=True))


# --- serving loop ---------------------------------------------------------------

@pytest.mark.parametrize("policy,max_cells,prec", [("fifo", 0, "f32c"), ("shortest", 12000, "f32c"),
                                                   ("shortest", 12000, "f64")])
def test_serve_stream_matches_alone(policy, max_cells, prec):
    """Every request of a stream finishes at its t_end with the state the
    same grid reaches alone, bit for bit, whatever joined it on the device;
    with a cell cap the live instances never hold more than the cap (but
    one)."""
    rng = np.random.default_rng(0)
    reqs, cases = [], []
    t = 0.0
    for k in range(12):
        t += rng.exponential(1 / 200.0)
        n = int(rng.choice([32, 48, 64, 80]))
        d, c = _desc(n, 500 + k, float(rng.uniform(0.02, 0.06)))
        reqs.append((t, d))
        cases.append(c)
    res, wall = F.serve_run(reqs, precision=prec, steps_per_round=4, policy=policy, max_cells=max_cells,
                            keep_results=True)
    assert all(r["status"] == 0 and r["finished"] >= r["admitted"] >= 0 for r in res)
    for (arr, d), r, c in zip(reqs, res, cases):
        assert r["admitted"] >= arr - 1e-3
        assert abs(r["t"] - d.t_end) <= 1e-12
        s = F.Solver(d.n, precision=prec, bc="transmissive", cfl=0.5)
        s.init_case(c)
        s.advance(d.t_end)
        assert s.sync().steps == r["steps"]
        assert np.array_equal(r["state"], s.get_state(interior=True))
        s.close()
    if max_cells:
        # at every admission the cells already live plus the newcomer's fit
        # the cap, unless nothing else was live
        for i, (_, d) in enumerate(reqs):
            live = sum(reqs[j][1].n ** 2 for j, o in enumerate(res)
                       if j != i and o["admitted"] <= res[i]["admitted"] < o["finished"])
            assert live == 0 or live + d.n ** 2 <= max_cells, (i, live)
    lat = sorted(r["finished"] - r["arrival"] for r in res)
    print("serve %s %s: %d requests in %.3f s, p50 %.4f s p99 %.4f s" % (policy, prec, len(res), wall,
                                                                           lat[len(lat) // 2], lat[-1]))


def test_solvers_on_concurrent_host_threads():
    """One solver per host thread (the C ABI's threading rule): solvers of
    every kernel family, created and stepped on four threads at once -- each
    setting up its kernels for the first time -- give the results they give
    one after another."""
    import threading

    specs = [dict(flux="up_ducros", precision="f64", order=9), dict(flux="keep"),
             dict(flux="rec3", bc="periodic"), dict(flux="up_hllc_d2av", order=9)]

    def run(spec):
        kw = dict(spec)
        kw.setdefault("bc", "reflect")
        s = F.Solver(48, **kw)
        s.init_case("sod")
        s.step(10)
        s.sync()
        out = s.get_state(interior=True)
        s.close()
        return out

    got, errors = [None] * len(specs), []

    def worker(k):
        try:
            got[k] = run(specs[k])
        except Exception as e:  # reported below, on the main thread
            errors.append(e)

    threads = [threading.Thread(target=worker, args=(k,)) for k in range(len(specs))]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors, errors
    for k, spec in enumerate(specs):
        assert np.array_equal(got[k], run(spec), equal_nan=True), spec
