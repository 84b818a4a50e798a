"""Whole-loop parity of the fused GPU turn against the oracle.

With quantum-excitation draws generated on the host and fed to both sides,
per-particle (z, ΔE) must agree within 1e-12 relative at EVERY turn of a
100-turn run of the 1e5-particle benchmark bunch (4096 bins), E0 likewise,
and the device bin counts must equal the oracle's histogram of the same
positions bit for bit.
"""
import math

import numpy as np
import pytest
import torch

from haissinskijulia_b200 import (BinGrid, HaissinskiError, Particles, ResidentBunch, WakeModel,
                                  benchmark_ring, create_simulation_buffers, longitudinal_evolve,
                                  reference_ring, synthetic_bunch)
from gpu_util import RTOL, assert_close, device_pair

pytestmark = pytest.mark.gpu


def _shared_grid(oracle, z0, cfg):
    return BinGrid.make(oracle.global_std(z0), cfg.nbins, cfg.wake.half_width_sigmas)


def run_turn_by_turn(gpu_ctx, oracle, cfg, n, turns, seed, check_every=1):
    bunch0 = synthetic_bunch(n, cfg.sigma_z, cfg.sigma_E, seed)
    z0, dE0 = bunch0.coordinates.z, bunch0.coordinates.dE
    draws = np.random.default_rng(seed + 1).normal(size=(turns, n))
    grid = _shared_grid(oracle, z0, cfg) if cfg.params.use_wakefield else None

    dz, de = device_pair(z0, dE0)
    ddraws = torch.from_numpy(draws).cuda()
    b = ResidentBunch(gpu_ctx, dz.data_ptr(), de.data_ptr(), n, cfg.params, cfg.nbins,
                      wake=cfg.wake, grid=grid, seed=seed)
    b.set_draws(ddraws.data_ptr(), 1, turns)

    zo, eo = z0.copy(), dE0.copy()
    st = oracle.state(zo, eo, cfg.params.to_c(), cfg.wake.to_c(), cfg.nbins,
                      grid.to_c() if grid is not None else None)
    zout, eout = torch.empty_like(dz), torch.empty_like(de)
    worst = {"z": 0.0, "dE": 0.0, "E0": 0.0}
    sz, se = cfg.sigma_z, cfg.sigma_E
    for t in range(1, turns + 1):
        b.advance(1)
        assert st.turn(np.ascontiguousarray(draws[t - 1])) == 0
        if t % check_every and t != turns:
            continue
        r = b.observe(zout.data_ptr(), eout.data_ptr())
        zg, eg = zout.cpu().numpy(), eout.cpu().numpy()
        worst["z"] = max(worst["z"], assert_close(zg, zo, sz, what=f"z turn {t}"))
        worst["dE"] = max(worst["dE"], assert_close(eg, eo, se, what=f"dE turn {t}"))
        e = abs(r.E0 - st.E0) / st.E0
        worst["E0"] = max(worst["E0"], e)
        assert e <= RTOL, f"E0 turn {t}: {e:.3e}"
        if cfg.params.use_wakefield:
            counts = b.histogram()
            assert np.array_equal(counts, oracle.histogram(zg, grid.to_c())), f"counts turn {t}"
            assert np.array_equal(counts, st.counts()), f"counts vs oracle bunch, turn {t}"
    res = b.finish()
    ro = st.result()
    assert res.sigma_E == pytest.approx(ro.sigma_E, rel=1e-12)
    assert res.sigma_z == pytest.approx(ro.sigma_z, rel=1e-12)
    assert res.sigma_E0_initial == pytest.approx(ro.sigma_E0_initial, rel=1e-14)
    assert res.sigma_z0_initial == pytest.approx(ro.sigma_z0_initial, rel=1e-14)
    # finish() left the device arrays at the same turn-boundary state
    assert_close(dz.cpu().numpy(), zo, sz, what="final z")
    assert_close(de.cpu().numpy(), eo, se, what="final dE")
    b.close()
    return worst


def test_benchmark_bunch_100_turns(gpu_ctx, oracle):
    """1e5 particles, 100 turns, 4096 bins, all physics on (the CPU-runnable config)."""
    cfg = benchmark_ring(n_turns=100, nbins=4096)
    worst = run_turn_by_turn(gpu_ctx, oracle, cfg, 100_000, 100, seed=2024)
    print("worst relative errors over 100 turns:", worst)


def test_reference_ring_reference_wake(gpu_ctx, oracle):
    """The reference's own benchmark ring and hard-coded wake (particle_factor current)."""
    cfg = reference_ring(100_000, n_turns=30)
    run_turn_by_turn(gpu_ctx, oracle, cfg, 100_000, 30, seed=1234)


@pytest.mark.parametrize("layout", [0, 1, 2, 3, 4, 5, 8, 9, 10, 11, 12, 13])
def test_thread_layouts(oracle, layout):
    """Every thread layout of the fused pass, with 16-bit (0-5) or 32-bit (8-13)
    bin counters, keeps per-particle parity and bit-exact counts."""
    from haissinskijulia_b200 import Context
    ctx = Context(0)
    ctx.set_pass_layout(layout)
    cfg = benchmark_ring(n_turns=20, nbins=4096)
    run_turn_by_turn(ctx, oracle, cfg, 100_003, 20, seed=40 + layout, check_every=4)


@pytest.mark.parametrize("flag", ["use_wakefield", "update_E0", "update_eta", "SR_damping",
                                  "use_excitation"])
def test_physics_switches(gpu_ctx, oracle, flag):
    cfg = benchmark_ring(n_turns=20, nbins=1024)
    cfg.params = cfg.params.replace(**{flag: False})
    run_turn_by_turn(gpu_ctx, oracle, cfg, 20_001, 20, seed=7, check_every=5)


def test_far_particles_take_the_reduced_rf_path(gpu_ctx, oracle):
    """Particles far from the synchronous one (|z k| > π/4, outside the bins)
    go through the fused pass's argument reduction of the RF kick; they must
    match the oracle's sin() like the rest of the bunch."""
    cfg = benchmark_ring(n_turns=3, nbins=1024)
    n = 4099
    p = synthetic_bunch(n, cfg.sigma_z, cfg.sigma_E, 77)
    far = np.array([0.05, -0.05, 0.0749, 0.0751, -0.0751, 0.1, -0.15, 0.2, 0.5, -1.0, 3.0, -3.0])
    p.coordinates.z[::300][: far.size] = far
    draws = np.random.default_rng(9).normal(size=(3, n))
    grid = _shared_grid(oracle, p.coordinates.z, cfg)
    zo, eo = p.coordinates.z.copy(), p.coordinates.dE.copy()
    buf = create_simulation_buffers(n, cfg.nbins, ctx=gpu_ctx)
    longitudinal_evolve(p, cfg.params, buf, wake=cfg.wake, grid=grid, qe_draws=draws)
    rc, _ = oracle.evolve(zo, eo, cfg.params.to_c(), cfg.wake.to_c(), cfg.nbins, grid.to_c(),
                          np.ascontiguousarray(draws))
    assert rc == 0
    assert_close(p.coordinates.z, zo, cfg.sigma_z, what="z")
    assert_close(p.coordinates.dE, eo, cfg.sigma_E, what="dE")


def test_crowded_bin_overflows_the_16bit_counters(gpu_ctx, oracle):
    """6e6 particles share one bin (every block deposits > 2^15 counts into it),
    so the pass's 16-bit shared counters overflow into the global array; the
    counts stay bit-exact and the bunch keeps per-particle parity."""
    cfg = benchmark_ring(n_turns=3, nbins=256)
    cfg.params.use_excitation = False
    n = 6_000_000
    rng = np.random.default_rng(5)
    z0 = np.zeros(n)
    dE0 = np.zeros(n)
    m = n // 100                      # a Gaussian 1 % keeps σ_z finite
    z0[:m] = rng.normal(0.0, cfg.sigma_z, m)
    dE0[:m] = rng.normal(0.0, cfg.sigma_E, m)
    grid = BinGrid.make(cfg.sigma_z, cfg.nbins, cfg.wake.half_width_sigmas)
    dz, de = device_pair(z0, dE0)
    b = ResidentBunch(gpu_ctx, dz.data_ptr(), de.data_ptr(), n, cfg.params, cfg.nbins,
                      wake=cfg.wake, grid=grid, seed=1)
    zo, eo = z0.copy(), dE0.copy()
    st = oracle.state(zo, eo, cfg.params.to_c(), cfg.wake.to_c(), cfg.nbins, grid.to_c())
    zout, eout = torch.empty_like(dz), torch.empty_like(de)
    for t in range(1, 4):
        b.advance(1)
        assert st.turn(None) == 0
        b.observe(zout.data_ptr(), eout.data_ptr())
        zg, eg = zout.cpu().numpy(), eout.cpu().numpy()
        counts = b.histogram()
        assert counts.max() >= n - m, "the crowded bin must hold the cold particles"
        assert np.array_equal(counts, oracle.histogram(zg, grid.to_c())), f"counts turn {t}"
        assert np.array_equal(counts, st.counts()), f"counts vs oracle bunch, turn {t}"
        assert_close(zg, zo, cfg.sigma_z, what=f"z turn {t}")
        assert_close(eg, eo, cfg.sigma_E, what=f"dE turn {t}")
    b.close()


@pytest.mark.parametrize("n", [2, 3, 5, 31, 33, 1001])
def test_tiny_bunches(gpu_ctx, oracle, n):
    cfg = benchmark_ring(n_turns=6, nbins=64)
    run_turn_by_turn(gpu_ctx, oracle, cfg, n, 6, seed=n)


def test_longitudinal_evolve_host_api(gpu_ctx, oracle):
    """The drop-in longitudinal_evolve (host buffers in, tuple out) vs or_evolve."""
    cfg = benchmark_ring(n_turns=40, nbins=2048)
    n = 50_001
    p0 = synthetic_bunch(n, cfg.sigma_z, cfg.sigma_E, 99)
    draws = np.random.default_rng(5).normal(size=(40, n))
    grid = _shared_grid(oracle, p0.coordinates.z, cfg)
    p = p0.copy()
    buf = create_simulation_buffers(n, cfg.nbins, ctx=gpu_ctx)
    sE, sz, E0 = longitudinal_evolve(p, cfg.params, buf, wake=cfg.wake, grid=grid, qe_draws=draws)
    zo, eo = p0.coordinates.z.copy(), p0.coordinates.dE.copy()
    rc, ro = oracle.evolve(zo, eo, cfg.params.to_c(), cfg.wake.to_c(), cfg.nbins, grid.to_c(),
                           np.ascontiguousarray(draws))
    assert rc == 0
    assert_close(p.coordinates.z, zo, cfg.sigma_z, what="z")
    assert_close(p.coordinates.dE, eo, cfg.sigma_E, what="dE")
    assert (sE, sz, E0) == pytest.approx((ro.sigma_E, ro.sigma_z, ro.E0), rel=1e-12)


def test_library_grid_matches_oracle_grid(gpu_ctx, oracle):
    """Without an explicit grid both sides build it from their own σ_z0."""
    cfg = benchmark_ring(n_turns=3, nbins=4096)
    n = 65_536
    p0 = synthetic_bunch(n, cfg.sigma_z, cfg.sigma_E, 3)
    p = p0.copy()
    buf = create_simulation_buffers(n, cfg.nbins, ctx=gpu_ctx)
    r = longitudinal_evolve(p, cfg.params.replace(use_excitation=False), buf, wake=cfg.wake,
                            full_result=True)
    zo, eo = p0.coordinates.z.copy(), p0.coordinates.dE.copy()
    rc, ro = oracle.evolve(zo, eo, cfg.params.replace(use_excitation=False).to_c(),
                           cfg.wake.to_c(), cfg.nbins)
    assert rc == 0
    assert r.sigma_z0_initial == pytest.approx(ro.sigma_z0_initial, rel=1e-14)
    assert_close(p.coordinates.z, zo, cfg.sigma_z, what="z")


def test_philox_runs_are_deterministic(gpu_ctx):
    cfg = benchmark_ring(n_turns=25, nbins=4096)
    n = 100_000
    outs = []
    for _ in range(2):
        p = synthetic_bunch(n, cfg.sigma_z, cfg.sigma_E, 11)
        buf = create_simulation_buffers(n, cfg.nbins, ctx=gpu_ctx)
        outs.append((longitudinal_evolve(p, cfg.params, buf, wake=cfg.wake, seed=42), p))
    assert outs[0][0] == outs[1][0]
    assert np.array_equal(outs[0][1].coordinates.z, outs[1][1].coordinates.z)
    assert np.array_equal(outs[0][1].coordinates.dE, outs[1][1].coordinates.dE)


def test_error_behaviour(gpu_ctx):
    cfg = benchmark_ring(n_turns=2, nbins=64)
    buf = create_simulation_buffers(10, 64, ctx=gpu_ctx)
    p = synthetic_bunch(10, cfg.sigma_z, cfg.sigma_E, 1)
    # nbins <= 0 (src/evolution.jl:264)
    with pytest.raises(HaissinskiError, match="HJ_ERR_NBINS"):
        longitudinal_evolve(p, cfg.params, buf.__class__(10, 0, ctx=gpu_ctx), wake=cfg.wake)
    # cτ <= 0 and pipe_radius <= 0 (src/evolution.jl:277-278)
    bad = WakeModel(cfg.wake.wake_factor, cfg.wake.wake_sqrt, 0.0)
    with pytest.raises(HaissinskiError, match="HJ_ERR_WAKE_PARAM"):
        longitudinal_evolve(p, cfg.params, buf, wake=bad)
    with pytest.raises(HaissinskiError, match="HJ_ERR_WAKE_PARAM"):
        longitudinal_evolve(p, cfg.params.replace(pipe_radius=0.0), buf, wake=cfg.wake)
    # zero particles with the wake on raises like the reference's log10(0) path
    empty = Particles(np.zeros(0), np.zeros(0))
    with pytest.raises(HaissinskiError, match="HJ_ERR_EMPTY"):
        longitudinal_evolve(empty, cfg.params, buf, wake=cfg.wake)
    # host-fed draws of the wrong size
    with pytest.raises(ValueError):
        longitudinal_evolve(p, cfg.params, buf, wake=cfg.wake, qe_draws=np.zeros(3))
    # more than the supported bins
    with pytest.raises(HaissinskiError, match="HJ_ERR_TOO_LARGE"):
        longitudinal_evolve(p, cfg.params, buf.__class__(10, 32768, ctx=gpu_ctx), wake=cfg.wake)
    # the context still works after the errors
    sE, sz, E0 = longitudinal_evolve(p, cfg.params, buf, wake=cfg.wake)
    assert math.isfinite(sE) and math.isfinite(E0)


def test_single_particle_has_zero_spread(gpu_ctx, oracle):
    cfg = benchmark_ring(n_turns=3, nbins=16)
    p = Particles(np.array([1e-3]), np.array([1e5]))
    buf = create_simulation_buffers(1, 16, ctx=gpu_ctx)
    params = cfg.params.replace(use_wakefield=False)
    r = longitudinal_evolve(p, params, buf, wake=cfg.wake, full_result=True)
    assert r.sigma_E == 0.0 and r.sigma_z == 0.0 and r.sigma_z0_initial == 0.0
    zo, eo = np.array([1e-3]), np.array([1e5])
    rc, ro = oracle.evolve(zo, eo, params.to_c(), cfg.wake.to_c(), 16)
    assert rc == 0 and r.E0 == pytest.approx(ro.E0, rel=1e-15)
    assert p.coordinates.z[0] == pytest.approx(zo[0], rel=1e-12)


def test_single_particle_with_wake(gpu_ctx, oracle):
    """One particle: σ_z0 = 0 so the bins shrink to ±1e-6 m (src/evolution.jl:272)
    and the wake current (src/evolution.jl:386) is 0/0 = NaN.  A particle outside
    the bins sees a zero potential and stays finite, as in the reference; one
    inside turns the bunch NaN in the reference, which the library reports as
    HJ_ERR_NONFINITE."""
    cfg = benchmark_ring(n_turns=2, nbins=16)
    buf = create_simulation_buffers(1, 16, ctx=gpu_ctx)
    zo, eo = np.array([1e-3]), np.array([1e5])
    rc, ro = oracle.evolve(zo, eo, cfg.params.to_c(), cfg.wake.to_c(), 16)
    assert rc == 0 and math.isfinite(ro.E0)
    p = Particles(np.array([1e-3]), np.array([1e5]))
    r = longitudinal_evolve(p, cfg.params, buf, wake=cfg.wake, full_result=True)
    assert r.E0 == pytest.approx(ro.E0, rel=1e-12)
    assert p.coordinates.dE[0] == pytest.approx(eo[0], rel=1e-12)

    # at rest on the synchronous particle (no QE): z stays 0, inside the bins
    quiet = cfg.params.replace(use_excitation=False)
    zo, eo = np.array([0.0]), np.array([0.0])
    rc, ro = oracle.evolve(zo, eo, quiet.to_c(), cfg.wake.to_c(), 16)
    assert rc == 0 and math.isnan(ro.E0)
    p = Particles(np.array([0.0]), np.array([0.0]))
    with pytest.raises(HaissinskiError, match="HJ_ERR_NONFINITE"):
        longitudinal_evolve(p, quiet, buf, wake=cfg.wake)


def test_invalid_pass_layouts_are_refused(gpu_ctx):
    from haissinskijulia_b200 import Context, HaissinskiError
    from haissinskijulia_b200 import _lib
    ctx = Context(0)
    for bad in (-2, 6, 7, 14, 15, 22, 30, 32):
        with pytest.raises(HaissinskiError) as e:
            ctx.set_pass_layout(bad)
        assert e.value.status == _lib.HJ_ERR_ARG
    for good in (-1, 0, 4, 5, 8, 12, 13, 16, 23, 24, 29):
        ctx.set_pass_layout(good)
    ctx.close()
