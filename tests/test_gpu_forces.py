"""GPU force parity through the C ABI against the oracle and the reference.

Tolerances (written per test):
  * FP64 kernel: per-particle relative error <= 1e-12 against the reference's
    double-precision forces and the extended-precision oracle (only summation
    order and the reciprocal square root's rounding differ);
  * FP32C kernel: median per-particle relative error <= 1e-6 against the
    extended-precision oracle, with a stated bound on the worst particle.
"""
import os

import numpy as np
import pytest

from conftest import golden, rel_err

pytestmark = pytest.mark.gpu

FP64, FP32C = 0, 1


def upload(ctx, s):
    ctx.upload({k: s[k] for k in ("x", "y", "z", "m")} | {k: s.get(k) for k in ("vx", "vy", "vz")})


def truth(oracle, s, eps2, G=1.0):
    return oracle.accel(s["x"], s["y"], s["z"], s["m"], G=G, eps2=eps2, extended=True)


@pytest.mark.parametrize("name", ["ref_forces_random_n1000.npz", "ref_forces_plummer_n2048.npz"])
def test_fp64_matches_reference_golden(ctx, name):
    g = golden(name)
    ctx.upload({"x": g["x"], "y": g["y"], "z": g["z"], "m": g["m"]})
    F = ctx.forces(FP64, G=1.0, eps2=0.0, want_force=True)
    for key in [k for k in g if k.startswith("F_")]:
        assert rel_err(F, g[key]).max() <= 1e-12, key


def test_fp64_ring_known_answer(ctx):
    g = golden("ref_ring_n1001.npz")
    ctx.upload({k: g[k] for k in ("x", "y", "z", "m")})
    F = ctx.forces(FP64, want_force=True)
    assert rel_err(F[:, :-1], g["F_analytic"][:, :-1]).max() <= 1e-11
    assert rel_err(F[:, :-1], g["F_simple"][:, :-1]).max() <= 1e-12
    assert np.abs(F[:, -1]).max() <= 1e-9 * np.abs(g["F_analytic"]).max()


@pytest.mark.parametrize("ic,n,eps", [("plummer", 2048, 1e-3), ("ball", 4096, 1e-2),
                                      ("plummer", 5000, 0.0), ("twocomp", 6000, 1e-3)])
def test_fp64_matches_oracle(ctx, nbr, oracle, ic, n, eps):
    s = {"plummer": lambda: nbr.plummer(n, 0), "ball": lambda: nbr.uniform_ball(n, 1),
         "twocomp": lambda: nbr.two_component(n, n // 100, 1000.0, 4)}[ic]()
    upload(ctx, s)
    a = ctx.forces(FP64, eps2=eps * eps)
    assert rel_err(a, truth(oracle, s, eps * eps)).max() <= 1e-12


@pytest.mark.parametrize("ic,n,eps,worst", [("plummer", 8192, 1e-3, 1e-4), ("ball", 8192, 1e-2, 1e-4),
                                            ("twocomp", 8192, 1e-3, 1e-4)])
def test_fp32c_accuracy(ctx, nbr, oracle, ic, n, eps, worst):
    s = {"plummer": lambda: nbr.plummer(n, 2), "ball": lambda: nbr.uniform_ball(n, 1),
         "twocomp": lambda: nbr.two_component(n, n // 100, 1000.0, 4)}[ic]()
    upload(ctx, s)
    a = ctx.forces(FP32C, eps2=eps * eps)
    err = rel_err(a, truth(oracle, s, eps * eps))
    assert np.median(err) <= 1e-6, np.median(err)
    assert err.max() <= worst, err.max()


def test_fp32c_offset_system_keeps_accuracy(ctx, nbr, oracle):
    """Tile-relative coordinates: a system far from the origin loses nothing."""
    s = nbr.plummer(4096, 5)
    for k, d in (("x", 1.0e3), ("y", -2.0e3), ("z", 5.0e2)):
        s[k] = s[k] + d
    upload(ctx, s)
    err = rel_err(ctx.forces(FP32C, eps2=1e-6), truth(oracle, s, 1e-6))
    assert np.median(err) <= 1e-6 and err.max() <= 1e-4


@pytest.mark.parametrize("n", [1, 2, 3, 31, 32, 33, 127, 128, 129, 255, 1023, 1024, 1025, 3001])
@pytest.mark.parametrize("prec", [FP64, FP32C])
def test_edge_sizes(ctx, nbr, oracle, n, prec):
    s = nbr.plummer(n, 100 + n)
    upload(ctx, s)
    a = ctx.forces(prec, eps2=1e-4)
    if n == 1:
        assert np.all(a == 0.0)
        return
    err = rel_err(a, truth(oracle, s, 1e-4))
    if prec == FP64:
        assert err.max() <= 1e-12
    else:
        assert np.median(err) <= 1e-6 and err.max() <= 1e-4


@pytest.mark.parametrize("prec", [FP64, FP32C])
def test_every_kernel_configuration_agrees(ctx, nbr, oracle, prec):
    s = nbr.plummer(6000, 17)
    upload(ctx, s)
    ref = truth(oracle, s, 1e-6)
    # (1, F): the small-N warp-splitting kernel with F lane groups per warp;
    # (3, 8): the Newton-3 kernel
    cfgs = [(4, 2), (4, 4), (4, 8), (8, 2), (8, 4), (1, 2), (1, 4), (1, 8), (3, 8)]
    if prec == FP32C:
        cfgs.append((3, 16))  # Newton-3, two warps per row block
    for ni, warps in cfgs:
        for split in (1, 3, 0, 47):
            ctx.set_force_config(prec, ni, warps, split)
            err = rel_err(ctx.forces(prec, eps2=1e-6), ref)
            if prec == FP64:
                assert err.max() <= 1e-12, (ni, warps, split)
            else:
                assert np.median(err) <= 1e-6 and err.max() <= 1e-4, (ni, warps, split)
    ctx.set_force_config(prec, 0)


@pytest.mark.parametrize("prec", [FP64, FP32C])
def test_deterministic(ctx, nbr, prec):
    s = nbr.plummer(20000, 3)
    upload(ctx, s)
    a = ctx.forces(prec, eps2=1e-6)
    b = ctx.forces(prec, eps2=1e-6)
    np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("prec", [FP64, FP32C])
def test_accel_ij_separate_sets(ctx, nbr, oracle, prec):
    src = nbr.plummer(3000, 41)
    rcv = nbr.uniform_ball(777, 42)
    a = ctx.accel_ij(rcv["x"], rcv["y"], rcv["z"], src["x"], src["y"], src["z"], src["m"],
                     precision=prec, eps2=1e-6)
    # Oracle: receivers as zero-mass members of the combined system.
    comb = {k: np.concatenate([src[k], rcv[k]]) for k in ("x", "y", "z")}
    comb["m"] = np.concatenate([src["m"], np.zeros(777)])
    ref = oracle.accel_subset(comb["x"], comb["y"], comb["z"], comb["m"], np.arange(3000, 3777), eps2=1e-6)
    err = rel_err(a, ref)
    if prec == FP64:
        assert err.max() <= 1e-12
    else:
        assert np.median(err) <= 1e-6


def test_want_force_and_G(ctx, nbr):
    s = nbr.two_component(4000, 40, 1000.0, 9)
    upload(ctx, s)
    a = ctx.forces(FP64, G=1.0, eps2=1e-6)
    F = ctx.forces(FP64, G=2.5, eps2=1e-6, want_force=True)
    np.testing.assert_allclose(F, 2.5 * a * s["m"], rtol=1e-15, atol=0)


def test_zero_mass_particles_exert_nothing(ctx, nbr, oracle):
    s = nbr.plummer(2000, 12)
    s["m"][::3] = 0.0
    upload(ctx, s)
    a = ctx.forces(FP64, eps2=1e-6)
    assert rel_err(a, truth(oracle, s, 1e-6)).max() <= 1e-12


@pytest.mark.parametrize("prec", [FP64, FP32C])
def test_unsoftened_coincident_pair_is_skipped(ctx, prec):
    x = np.array([0.0, 0.0, 1.0]); y = np.zeros(3); z = np.zeros(3); m = np.ones(3)
    ctx.upload({"x": x, "y": y, "z": z, "m": m})
    a = ctx.forces(prec, eps2=0.0)
    assert np.all(np.isfinite(a))
    np.testing.assert_allclose(a[0], [1.0, 1.0, -2.0], rtol=1e-6)


def test_invalid_inputs_are_rejected(ctx, nbr):
    s = nbr.plummer(100, 1)
    bad = dict(s)
    bad["x"] = s["x"].copy()
    bad["x"][7] = np.nan
    with pytest.raises(nbr.NbrError) as ei:
        ctx.upload(bad)
    assert ei.value.status == 7
    neg = dict(s)
    neg["m"] = s["m"].copy()
    neg["m"][3] = -1.0
    with pytest.raises(nbr.NbrError) as ei:
        ctx.upload(neg)
    assert ei.value.status == 1
    # a rejected upload leaves no system behind
    with pytest.raises(nbr.NbrError) as ei:
        ctx.forces(FP64, eps2=0.0)
    assert ei.value.status == 5
    inf_v = dict(s)
    inf_v["vz"] = s["vz"].copy()
    inf_v["vz"][99] = np.inf
    with pytest.raises(nbr.NbrError) as ei:
        ctx.upload(inf_v)
    assert ei.value.status == 7
    upload(ctx, s)
    with pytest.raises(nbr.NbrError):
        ctx.forces(FP64, eps2=-1.0)
    with pytest.raises(nbr.NbrError):
        ctx.forces(7, eps2=0.0)


def test_no_system_uploaded(nbr):
    with nbr.Context(0) as c:
        with pytest.raises(nbr.NbrError) as ei:
            c.forces(FP64)
        assert ei.value.status == 5


@pytest.mark.parametrize("prec", [FP64, FP32C])
def test_bounded_wait_expires_cleanly(nbr, oracle, prec):
    """A tile copy that is never issued makes the bounded wait expire: the call
    returns NBR_ERR_TIMEOUT and the context stays usable."""
    s = nbr.plummer(4096, 77)
    with nbr.Context(0) as c:
        upload(c, s)
        os.environ["NBR_WAIT_LIMIT_MS"] = "100"
        os.environ["NBR_TEST_SKIP_TILE"] = "1"
        try:
            with pytest.raises(nbr.NbrError) as ei:
                c.forces(prec, eps2=1e-6)
            assert ei.value.status == 4
        finally:
            del os.environ["NBR_TEST_SKIP_TILE"]
            del os.environ["NBR_WAIT_LIMIT_MS"]
        err = rel_err(c.forces(prec, eps2=1e-6), truth(oracle, s, 1e-6))
        assert (err.max() if prec == FP64 else np.median(err)) <= (1e-12 if prec == FP64 else 1e-6)


def test_potential_and_diagnostics(ctx, nbr, oracle):
    g = golden("ref_energy_plummer_n2048.npz")
    ctx.upload({k: g[k] for k in ("x", "y", "z", "vx", "vy", "vz", "m")})
    U = ctx.potential(eps2=0.0)
    assert abs(U - g["U_scalar"]) <= 1e-12 * abs(g["U_scalar"])
    d = ctx.diagnostics(eps2=0.0)
    assert abs(d["T"] - g["T"]) <= 1e-13 * g["T"]
    s = nbr.plummer(3000, 4)
    upload(ctx, s)
    U, phi = ctx.potential(eps2=1e-6, per_particle=True)
    ref_phi = oracle.potential(s["x"], s["y"], s["z"], s["m"], eps2=1e-6)
    np.testing.assert_allclose(phi, ref_phi, rtol=1e-12)
    e = oracle.energy(s, eps2=1e-6)
    d = ctx.diagnostics(eps2=1e-6)
    assert abs(d["E"] - e["E"]) <= 1e-12 * abs(e["E"])
    np.testing.assert_allclose(d["P"], e["P"], atol=1e-14)
    np.testing.assert_allclose(d["L"], e["L"], atol=1e-14)
    assert abs(d["M"] - 1.0) < 1e-13


# Worst-particle bound of the FP32C kernels at full size, against the
# extended-precision oracle.  The error of the worst particles comes from
# close pairs: source and receiver coordinates are rounded to FP32 relative to
# the FP64 origin of the source tile (a tile is 128 particles in index order,
# so it spans the system), and for a pair much closer than that distance the
# rounding of the two coordinates is a large fraction of their difference.
# Accumulation is not the cause: summing the same FP32 pair terms in FP64
# changes the worst errors by under 10 %.  The median stays near 4e-8.
FP32C_WORST = {262144: 5e-4, 1048576: 2e-3}


@pytest.mark.parametrize("n,seed", [(262144, 2), (1048576, 2)])
def test_full_size_plummer_sampled(ctx, nbr, oracle, n, seed):
    """Full-size Plummer systems: random receivers and the 64 worst particles
    of the FP32C-vs-FP64 comparison over all particles, against the
    extended-precision oracle; Newton's third law over all particles."""
    s = nbr.plummer(n, seed)
    upload(ctx, s)
    eps2 = 1e-6
    a64 = ctx.forces(FP64, eps2=eps2)
    a32 = ctx.forces(FP32C, eps2=eps2)
    eall = rel_err(a32, a64)
    assert np.median(eall) <= 1e-6
    rnd = np.random.default_rng(0).choice(n, 192, replace=False)
    worst = np.argsort(eall)[-64:]
    idx = np.concatenate([rnd, worst])
    ref = oracle.accel_subset(s["x"], s["y"], s["z"], s["m"], idx, eps2=eps2)
    # FP64 is exact to 1e-12 on every sampled particle, the worst included,
    # so the FP32C-vs-FP64 error is the FP32C kernel's own
    assert rel_err(a64[:, idx], ref).max() <= 1e-12
    e32 = rel_err(a32[:, idx], ref)
    assert np.median(e32[:192]) <= 1e-6, np.median(e32[:192])
    assert e32.max() <= FP32C_WORST[n], e32.max()
    # total momentum change sum m a ~ 0 relative to sum m |a|
    for a in (a64, a32):
        net = np.abs((a * s["m"]).sum(axis=1)).max()
        assert net <= 1e-6 * (np.linalg.norm(a, axis=0) * s["m"]).sum()


@pytest.mark.parametrize("prec", [FP64, FP32C])
def test_two_component_error_by_mass_class(ctx, nbr, oracle, prec):
    """The mass-ratio stress test's error, stratified by receiver and source
    mass class: each source class through nbr_accel_ij against the
    extended-precision oracle on sampled receivers of both classes."""
    n, nh, eps2 = 32768, 328, 1e-6
    s = nbr.two_component(n, nh, 1000.0, 4)
    rng = np.random.default_rng(7)
    idx = np.concatenate([rng.choice(nh, 64, replace=False), nh + rng.choice(n - nh, 448, replace=False)])
    heavy = np.zeros(n, dtype=bool)
    heavy[:nh] = True
    for src in (heavy, ~heavy):
        got = ctx.accel_ij(s["x"][idx], s["y"][idx], s["z"][idx], s["x"][src], s["y"][src], s["z"][src],
                           s["m"][src], precision=prec, eps2=eps2)
        # receivers as zero-mass copies in front of the source class
        X = {k: np.concatenate([s[k][idx], s[k][src]]) for k in ("x", "y", "z")}
        M = np.concatenate([np.zeros(len(idx)), s["m"][src]])
        ref = oracle.accel_subset(X["x"], X["y"], X["z"], M, np.arange(len(idx)), eps2=eps2)
        err = rel_err(got, ref)
        for cls in (slice(0, 64), slice(64, None)):  # heavy receivers, light receivers
            if prec == FP64:
                assert err[cls].max() <= 1e-12
            else:
                assert np.median(err[cls]) <= 1e-6 and err[cls].max() <= 1e-4


@pytest.mark.parametrize("n", [1, 3, 129, 20000])
def test_potential_sizes_and_self_term(ctx, nbr, oracle, n):
    """The tiled FP64 potential: ragged sizes, the split reduction (large n)
    and the self pair, which with eps > 0 would add m_i / eps if not skipped."""
    s = nbr.plummer(n, 14)
    upload(ctx, s)
    eps2 = 1e-2
    U, phi = ctx.potential(eps2=eps2, per_particle=True)
    ref = oracle.potential(s["x"], s["y"], s["z"], s["m"], eps2=eps2)
    if n == 1:
        assert phi[0] == 0.0 and U == 0.0
        return
    np.testing.assert_allclose(phi, ref, rtol=1e-12)
    assert abs(U - 0.5 * float(np.dot(s["m"], ref))) <= 1e-12 * abs(U)


@pytest.mark.parametrize("prec", [FP64, FP32C])
def test_small_kernel_leapfrog_and_ranges(ctx, nbr, oracle, prec):
    """The small-N kernel on the paths beyond nbr_forces: a KDK run (its
    epilogue packs no FP32C records, so every step repacks them) and a
    receiver range of the multi-GPU partition."""
    n, eps2 = 1500, 1e-6
    s = nbr.plummer(n, 21)
    upload(ctx, s)
    ctx.set_force_config(prec, 1, 8, 0)
    try:
        ctx.run(prec, 0, 2, 1e-3, 10, eps2=eps2)
        got = ctx.download()
        want = oracle.kdk(s, 1e-3, 10, eps2=eps2)
        for k in ("x", "y", "z", "vx", "vy", "vz"):
            assert np.abs(got[k] - want[k]).max() <= (1e-12 if prec == FP64 else 1e-6), k
        upload(ctx, s)
        v0 = {k: s[k].copy() for k in ("vx", "vy", "vz")}
        ctx.step_range(prec, 0, 256, 700, 1.0, 0.0, 1.0, eps2)  # v += a on [256, 956)
        ctx.synchronize()
        st = ctx.state_tensors()
        dv = np.stack([st[k][:n].cpu().numpy() - v0[k] for k in ("vx", "vy", "vz")])
        ref = truth(oracle, s, eps2)
        e = rel_err(dv[:, 256:956], ref[:, 256:956])
        assert (e.max() <= 1e-12) if prec == FP64 else (np.median(e) <= 1e-6)
        assert not dv[:, :256].any() and not dv[:, 956:].any()
    finally:
        ctx.set_force_config(prec, 0)


@pytest.mark.parametrize("warps", [8, 16])
@pytest.mark.parametrize("n", [300, 4097, 20000, 70000])
def test_newton3_kernel(ctx, nbr, oracle, n, warps):
    """The Newton-3 FP32C kernels (each unordered pair once, acting on both
    particles; one warp per 256-particle row block, or two): accuracy against
    the extended-precision oracle, bit-for-bit repeatability, near-exact
    momentum balance, and a leapfrog run (its epilogue runs in the reduction
    kernel, with the record pack)."""
    s = nbr.plummer(n, 23)
    upload(ctx, s)
    eps2 = 1e-6
    ctx.set_force_config(FP32C, 3, warps, 0)
    try:
        a = ctx.forces(FP32C, eps2=eps2)
        b = ctx.forces(FP32C, eps2=eps2)
        np.testing.assert_array_equal(a, b)
        idx = np.arange(0, n, max(1, n // 500))
        ref = oracle.accel_subset(s["x"], s["y"], s["z"], s["m"], idx, eps2=eps2)
        e = rel_err(a[:, idx], ref)
        assert np.median(e) <= 1e-6 and e.max() <= 1e-4, (np.median(e), e.max())
        net = np.abs((s["m"] * a).sum(axis=1)).max()
        scale = (s["m"] * np.linalg.norm(a, axis=0)).sum()
        assert net <= 1e-6 * scale
        if n <= 20000:
            upload(ctx, s)
            ctx.run(FP32C, 0, 2, 1e-3, 5, eps2=eps2)
            got = ctx.download()
            want = oracle.kdk(s, 1e-3, 5, eps2=eps2)
            for k in ("x", "y", "z", "vx", "vy", "vz"):
                assert np.abs(got[k] - want[k]).max() <= 1e-6, k
    finally:
        ctx.set_force_config(FP32C, 0)


@pytest.mark.parametrize("n,eps2", [(300, 1e-6), (4097, 1e-6), (20000, 1e-6), (70000, 1e-6),
                                    (300, 0.0), (4097, 0.0), (20000, 0.0)])
def test_newton3_kernel_fp64(ctx, nbr, oracle, n, eps2):
    """The Newton-3 FP64 kernel (set_force_config(FP64, 3, 8)): the FP64
    drop-in bound of 1e-12 against the extended-precision oracle, with and
    without softening (eps2 = 0 excludes the self pair), bit-for-bit
    repeatability, agreement with the plain FP64 kernel to summation order,
    momentum balance, and a KDK run through its reduction epilogue."""
    s = nbr.plummer(n, 29)
    upload(ctx, s)
    ctx.set_force_config(FP64, 3, 8, 0)
    try:
        assert ctx.get_force_config(FP64, eps2)[0] == 3
        a = ctx.forces(FP64, eps2=eps2)
        b = ctx.forces(FP64, eps2=eps2)
        np.testing.assert_array_equal(a, b)
        idx = np.arange(0, n, max(1, n // 500))
        ref = oracle.accel_subset(s["x"], s["y"], s["z"], s["m"], idx, eps2=eps2)
        e = rel_err(a[:, idx], ref)
        assert e.max() <= 1e-12, e.max()
        ctx.set_force_config(FP64, 4, 4, 0)
        plain = ctx.forces(FP64, eps2=eps2)
        assert rel_err(a, plain).max() <= 1e-12
        net = np.abs((s["m"] * a).sum(axis=1)).max()
        scale = (s["m"] * np.linalg.norm(a, axis=0)).sum()
        assert net <= 1e-12 * scale
        if n <= 20000 and eps2 > 0:
            ctx.set_force_config(FP64, 3, 8, 0)
            upload(ctx, s)
            ctx.run(FP64, 0, 2, 1e-3, 5, eps2=eps2)
            got = ctx.download()
            want = oracle.kdk(s, 1e-3, 5, eps2=eps2)
            for k in ("x", "y", "z", "vx", "vy", "vz"):
                assert np.abs(got[k] - want[k]).max() <= 1e-11, k
    finally:
        ctx.set_force_config(FP64, 0)


@pytest.mark.parametrize("n", [9216, 10240, 11264, 12288, 15360, 17408])
def test_default_kernel_between_8k_and_18k(ctx, nbr, oracle, n):
    """Sizes where the default switches between the large kernels and the
    Newton-3 kernel by the grid model's efficiency (and one just above
    16384): whichever it takes, every sampled receiver within the tolerances
    against the extended-precision oracle, FP64 and FP32C."""
    s = nbr.plummer(n, 31)
    upload(ctx, s)
    eps2 = 1e-6
    idx = np.random.default_rng(n).choice(n, 256, replace=False)
    ref = oracle.accel_subset(s["x"], s["y"], s["z"], s["m"], idx, eps2=eps2)
    a64 = ctx.forces(FP64, eps2=eps2)
    assert rel_err(a64[:, idx], ref).max() <= 1e-12
    a32 = ctx.forces(FP32C, eps2=eps2)
    e = rel_err(a32[:, idx], ref)
    assert np.median(e) <= 1e-6 and e.max() <= 1e-4, (np.median(e), e.max())
