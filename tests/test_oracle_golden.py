"""The oracle against the reference itself (no GPU).

tests/golden/*_small.npz were produced by tests/golden/make_golden.py, which runs the
reference's own CUDA update (built unmodified from its sources, oracle/build_ref.sh) stage by
stage on a seeded synthetic scene with the Philox draws injected. Each test feeds the
recorded stage inputs to the oracle and compares with the recorded reference outputs:
bit-exact for indices, orderings, slots, ancestors and every value the reference forms with
FP32 operations the oracle mirrors; within a stated tolerance where the oracle evaluates in
FP64 what the reference accumulates in FP32.
"""
from pathlib import Path

import numpy as np
import pytest

from k3dom_b200 import _native as N
from oracle import binding as O

GOLD = Path(__file__).resolve().parent / "golden"
VARIANTS = ["k3dom", "dsphdmib"]


def load(variant):
    path = GOLD / f"{variant}_small.npz"
    if not path.exists():
        pytest.skip(f"{path.name} not generated")
    f = np.load(path)
    p = N.Params.from_buffer_copy(f["params"].tobytes())
    return f, p


def frames(f):
    return sorted({int(k[1:k.index("_")]) for k in f.files if k.startswith("f") and k[1].isdigit()})


def steady_frames(f):
    return [i for i in frames(f) if i > 0]


def particles(f, key):
    return {k: f[f"{key}_{k}"] for k in ("pos", "vel", "weight", "cell", "associated")}


# ------------------------------------------------------------------ draws
def test_philox_known_answers():
    # Random123 Philox4x32-10 known-answer vectors (Salmon et al., SC'11)
    assert list(O.philox_raw([0, 0, 0, 0], [0, 0])) == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
    assert list(O.philox_raw([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2)) == [0x408F276D, 0x41C83B0E, 0xA20BC7C6,
                                                                     0x6D5451FD]
    assert list(O.philox_raw([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0])) == [
        0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]


@pytest.mark.parametrize("variant", VARIANTS)
def test_uniform_draws_equal(variant):
    f, p = load(variant)
    P, B = int(f["P"]), int(f["B"])
    np.testing.assert_array_equal(O.uniforms(p.seed, 0, 2, 0, P), f["f0_init_uniforms"])
    for fr in steady_frames(f):
        np.testing.assert_array_equal(O.uniforms(p.seed, fr, 3, 0, B), f[f"f{fr}_birth_uniforms"])


@pytest.mark.parametrize("variant", VARIANTS)
def test_normals_close_to_libm(variant):
    f, p = load(variant)
    fr = steady_frames(f)[0]
    n = O.oracle()
    ref = f[f"f{fr}_normals"].reshape(-1)
    mine = np.empty_like(ref)
    n.orc_normals_libm(p.seed, fr, 0, ref.size // 6, mine)
    np.testing.assert_allclose(mine, ref, rtol=2e-6, atol=2e-6)


# ------------------------------------------------------------------ prediction and assignment
@pytest.mark.parametrize("variant", VARIANTS)
def test_predict_bit_exact(variant):
    f, p = load(variant)
    G, Gz = int(f["G"]), int(f["Gz"])
    for fr in steady_frames(f):
        out = O.predict(particles(f, f"f{fr}_pred_in"), f[f"f{fr}_normals"], G, Gz, float(f[f"f{fr}_dt"]),
                        p.persistence_prob, p.stddev_process_noise_position, p.stddev_process_noise_velocity,
                        p.init_max_velocity)
        ref = particles(f, f"f{fr}_pred_out")
        for k in ("pos", "vel", "weight", "cell"):
            np.testing.assert_array_equal(out[k], ref[k], err_msg=f"frame {fr} {k}")


@pytest.mark.parametrize("variant", VARIANTS)
def test_assignment_stable_order(variant):
    f, p = load(variant)
    C_ = int(f["G"]) ** 2 * int(f["Gz"])
    for fr in steady_frames(f):
        pr = particles(f, f"f{fr}_pred_out")
        perm, sk, st, en = O.assign(pr["cell"], C_)
        srt = particles(f, f"f{fr}_sorted")
        for k in ("pos", "vel", "weight", "cell"):
            np.testing.assert_array_equal(pr[k][perm], srt[k], err_msg=f"frame {fr} {k}")
        cells = f[f"f{fr}_cells_in"]
        np.testing.assert_array_equal(st, cells["start_idx"])
        np.testing.assert_array_equal(en, cells["end_idx"])


# ------------------------------------------------------------------ K3DOM mass update
def relerr(a, b, floor):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.abs(a - b) / np.maximum(np.abs(b), floor)


def k3dom_oracle_update(f, p, fr, cells_in):
    G, Gz = int(f["G"]), int(f["Gz"])
    C_ = G * G * Gz
    srt = particles(f, f"f{fr}_sorted") if fr > 0 else None
    if srt is not None:
        sw, swx, swy, swz = O.cell_sums(srt["cell"], srt["weight"], srt["vel"], C_)
        has = (cells_in["start_idx"] >= 0).astype(np.int32)
        dt = float(f[f"f{fr}_dt"])
    else:
        sw = swx = swy = swz = np.zeros(C_)
        has = np.zeros(C_, np.int32)
        dt = 0.0
    ev = O.bgki(G, Gz, p.resolution, f[f"f{fr}_sensor_rel"], p.ls, p.sigma, f[f"f{fr}_pts"])
    out = O.k3dom_update(dt, p.gamma, p.birth_prob, p.mass_scale, ev, cells_in["free_mass"],
                         cells_in["static_mass"], cells_in["dynamic_mass"], has, sw, swx, swy, swz)
    return ev, out


def dyn_pred32(f, fr, C_):
    """The reference's serial FP32 weight sum per cell (mass_update.cu:168-174)."""
    dp = np.zeros(C_, np.float32)
    if fr > 0:
        cells, w = f[f"f{fr}_sorted_cell"], f[f"f{fr}_sorted_weight"]
        for i in range(cells.size):
            dp[cells[i]] += w[i]
    return dp


def test_k3dom_fp32_mirror_matches_reference():
    """The oracle's FP32 restatement of BGKI and the mass update reproduces the reference's
    cells to 1e-5 (the residue is libm vs CUDA cospif/expf/powf in the last ulp)."""
    f, p = load("k3dom")
    G, Gz = int(f["G"]), int(f["Gz"])
    C_ = G * G * Gz
    for fr in frames(f):
        cin = f[f"f{fr}_cells_in"]
        cout = f[f"f{fr}_cells_occ"] if fr > 0 else f["f0_cells_out"]
        ev = O.bgki_ref32(G, Gz, p.resolution, f[f"f{fr}_sensor_rel"], p.ls, p.sigma, f[f"f{fr}_pts"])
        dt = float(f[f"f{fr}_dt"]) if fr > 0 else 0.0
        o = O.k3dom_update_ref32(dt, p.gamma, p.birth_prob, p.mass_scale, ev, cin["free_mass"],
                                 cin["static_mass"], cin["dynamic_mass"], dyn_pred32(f, fr, C_))
        for name, field in [("free", "free_mass"), ("static", "static_mass"), ("dyn", "dynamic_mass"),
                            ("pers", "pers_mass")]:
            e = relerr(o[name], cout[field], 1e-3)
            assert e.max() < 1e-5, (fr, name, e.max(), int(e.argmax()))
        assert relerr(o["born"], f[f"f{fr}_born"], 1e-3).max() < 1e-5


def test_k3dom_fp64_oracle_vs_reference_arithmetic():
    """FP64 evidence against the reference's FP32 formula: occupied evidence agrees to 1e-5;
    free evidence only to ~1e-3, because sqrt(d_c^2 - d_proj^2) (mass_update.cu:60) cancels in
    FP32, and where that radicand rounds negative the reference drops a whole term (NaN). The
    library evaluates the same distance in a well-conditioned form and is held to 1e-5 against
    FP64 (tests/test_gpu_parity.py)."""
    f, p = load("k3dom")
    G, Gz = int(f["G"]), int(f["Gz"])
    for fr in frames(f):
        ev32 = O.bgki_ref32(G, Gz, p.resolution, f[f"f{fr}_sensor_rel"], p.ls, p.sigma, f[f"f{fr}_pts"])
        ev64 = O.bgki(G, Gz, p.resolution, f[f"f{fr}_sensor_rel"], p.ls, p.sigma, f[f"f{fr}_pts"])
        ok = ev32["nan_drop"] == 0
        assert (~ok).sum() <= 3
        assert relerr(ev32["del_occ"], ev64["del_occ"], 1e-2 * p.sigma).max() < 1e-5
        assert relerr(ev32["del_free"], ev64["del_free"], 1e-2 * p.sigma)[ok].max() < 2e-3
        # the dropped terms are whole kernel values (up to sigma)
        drop = ev64["del_free"][~ok] - ev32["del_free"][~ok]
        assert np.all((drop > 0) & (drop <= p.sigma * 1.0001))


def test_k3dom_fp64_mass_update_consistent():
    """The FP64 mass update applied to the reference's own evidence reproduces its masses:
    the update equations (predict_mass, update_mass, separate_newborn_part) agree."""
    f, p = load("k3dom")
    G, Gz = int(f["G"]), int(f["Gz"])
    C_ = G * G * Gz
    for fr in frames(f):
        cin = f[f"f{fr}_cells_in"]
        cout = f[f"f{fr}_cells_occ"] if fr > 0 else f["f0_cells_out"]
        ev32 = O.bgki_ref32(G, Gz, p.resolution, f[f"f{fr}_sensor_rel"], p.ls, p.sigma, f[f"f{fr}_pts"])
        ev = {"del_occ": ev32["del_occ"].astype(np.float64), "del_free": ev32["del_free"].astype(np.float64)}
        has = (cin["start_idx"] >= 0).astype(np.int32) if fr > 0 else np.zeros(C_, np.int32)
        dp = dyn_pred32(f, fr, C_).astype(np.float64)
        z = np.zeros(C_)
        dt = float(f[f"f{fr}_dt"]) if fr > 0 else 0.0
        o = O.k3dom_update(dt, p.gamma, p.birth_prob, p.mass_scale, ev, cin["free_mass"], cin["static_mass"],
                           cin["dynamic_mass"], has, dp, z, z, z)
        for name, field in [("free", "free_mass"), ("static", "static_mass"), ("dyn", "dynamic_mass")]:
            assert relerr(cout[field], o[name], 1e-3).max() < 1e-5, (fr, name)
        # pers = dyn - born cancels when born ~ dyn: compare on the dynamic-mass scale
        scale = np.maximum(np.abs(o["dyn"]), 1e-3)
        assert (np.abs(cout["pers_mass"] - o["pers"]) / scale).max() < 1e-5


def test_k3dom_persistent_reweight_bit_exact():
    """updatePersistentParticlesKernel3 with p_A = 0: w' = mu_UA * w, and mu_UA = pers / pred."""
    f, p = load("k3dom")
    for fr in steady_frames(f):
        cells = f[f"f{fr}_cells_pers"]
        srt = particles(f, f"f{fr}_sorted")
        has = cells["start_idx"] >= 0
        pred = np.where(cells["pred_mass"] > 0, cells["pred_mass"], np.float32(1))
        mu = np.where(cells["pred_mass"] > 0, cells["pers_mass"] / pred, np.float32(0)).astype(np.float32)
        np.testing.assert_array_equal(cells["mu_UA"][has], mu[has])
        w = (np.float32(1.0) * cells["mu_UA"][srt["cell"]]) * srt["weight"]
        np.testing.assert_array_equal(f[f"f{fr}_reweighted"], w.astype(np.float32))


def subtract(cum, st, en):
    """include/common/common.h:20-28 in FP32."""
    lo = np.where(st > 0, cum[np.maximum(st - 1, 0)], np.float32(0))
    return np.where(st > 0, cum[en] - lo, cum[en]).astype(np.float32)


@pytest.mark.parametrize("variant", VARIANTS)
def test_moments_and_mu_from_reference_prefix_bit_exact(variant):
    """statisticalMomentsKernel2 and updatePersistentParticlesKernel2 restated on the
    reference's FP32 prefix arrays reproduce its mean velocities and mu_A. The prefix arrays
    come from a second thrust::inclusive_scan of the same data; CUB's float scan (decoupled
    look-back) is not run-to-run reproducible, so a few cells may differ from the reference's
    internal scan, by a few ulps of the running prefix."""
    f, p = load(variant)

    def check(got, acc, rho, cum_abs_max, what):
        exp = np.where(rho > 0, acc / np.where(rho > 0, rho, 1), np.float32(0)).astype(np.float32)
        same = got == exp
        assert same.mean() > 0.995, (what, same.mean())
        bound = 16 * cum_abs_max * 2.0 ** -23 / np.where(rho > 0, np.abs(rho), np.inf)
        assert np.all(np.abs(got.astype(np.float64) - exp) <= bound + 1e-6 * np.abs(exp)), what

    for fr in steady_frames(f):
        cells = f[f"f{fr}_cells_mom"]
        has = cells["start_idx"] >= 0
        st, en = cells["start_idx"][has], cells["end_idx"][has]
        rho = cells["pers_mass"][has]
        cum = f[f"f{fr}_wv_cum"]
        for k, fld in enumerate(("mean_x_vel", "mean_y_vel", "mean_z_vel")):
            check(cells[fld][has], subtract(cum[:, k], st, en), rho, np.abs(cum[:, k]).max(), (fr, fld))
            assert np.all(cells[fld][~has] == 0)
        pw_cum = f[f"f{fr}_postw_cum"]
        pw = subtract(pw_cum, st, en)
        got = f[f"f{fr}_cells_pers"]["mu_A"][has]
        exp = np.where(pw > 0, rho / np.where(pw > 0, pw, 1), np.float32(0)).astype(np.float32)
        assert (got == exp).mean() > 0.995


@pytest.mark.parametrize("variant", VARIANTS)
def test_mean_velocity_fp64_vs_reference(variant):
    """FP64 per-cell sums against the reference's prefix differences: they agree wherever the
    prefix difference is well conditioned; where a cell's |sum w v| is small against the running
    prefix, the reference's FP32 difference (statistical_moments.cu:12-20) loses digits and the
    disagreement is bounded by a few ulps of the prefix, divided by the cell's mass."""
    f, p = load(variant)
    C_ = int(f["G"]) ** 2 * int(f["Gz"])
    for fr in steady_frames(f):
        cells = f[f"f{fr}_cells_mom"]
        srt = particles(f, f"f{fr}_sorted")
        w = f[f"f{fr}_reweighted"]
        has = cells["start_idx"] >= 0
        pers = cells["pers_mass"].astype(np.float64)
        cum = f[f"f{fr}_wv_cum"]
        for k, fld in enumerate(("mean_x_vel", "mean_y_vel", "mean_z_vel")):
            s = np.zeros(C_)
            np.add.at(s, srt["cell"], (w * srt["vel"][:, k]).astype(np.float64))
            exp = np.where(has & (pers > 0), s / np.where(pers > 0, pers, 1), 0.0)
            got = cells[fld].astype(np.float64)
            ulp_prefix = np.abs(cum[:, k]).max() * 2.0 ** -23
            bound = 64 * ulp_prefix / np.where(pers > 0, pers, np.inf) + 1e-5 * np.abs(exp) + 1e-6
            assert np.all(np.abs(got - exp) <= bound), (fr, fld)


# ------------------------------------------------------------------ slots and ancestors
@pytest.mark.parametrize("variant", VARIANTS)
def test_first_frame_particles_bit_exact(variant):
    f, p = load(variant)
    P, G = int(f["P"]), int(f["G"])
    o = O.init_particles(f["f0_born_cum"], P, G, p.init_max_velocity, p.particle_min_vel, f["f0_init_uniforms"],
                         prev_cell=f["f0_prev_cell"])
    ref = particles(f, "f0_init")
    for k in ("cell", "pos", "vel", "weight"):
        np.testing.assert_array_equal(o[k], ref[k], err_msg=k)


@pytest.mark.parametrize("variant", VARIANTS)
def test_births_bit_exact(variant):
    f, p = load(variant)
    B, G = int(f["B"]), int(f["G"])
    for fr in steady_frames(f):
        o = O.births(f[f"f{fr}_born"], f[f"f{fr}_born_cum"], B, G, 0.0, p.init_max_velocity, p.particle_min_vel,
                     f[f"f{fr}_birth_uniforms"], prev_cell=f[f"f{fr}_birth_prev_cell"],
                     prev_assoc=f[f"f{fr}_birth_prev_assoc"])
        ref = particles(f, f"f{fr}_birth")
        for k in ("cell", "associated", "pos", "vel", "weight"):
            np.testing.assert_array_equal(o[k], ref[k], err_msg=f"frame {fr} {k}")


@pytest.mark.parametrize("variant", VARIANTS)
def test_penalty_bit_exact(variant):
    f, p = load(variant)
    m2 = np.float32(p.particle_min_vel) * np.float32(p.particle_min_vel)
    for fr in steady_frames(f):
        for w_before, vel, w_after in ((f[f"f{fr}_reweighted"], f[f"f{fr}_sorted_vel"], f[f"f{fr}_joint_sorted_w"]),
                                       (f[f"f{fr}_birth_weight"], f[f"f{fr}_birth_vel"], f[f"f{fr}_joint_birth_w"])):
            v = vel.astype(np.float32)
            sp = (v[:, 0] * v[:, 0] + v[:, 1] * v[:, 1]) + v[:, 2] * v[:, 2]
            np.testing.assert_array_equal(np.where(sp < m2, np.float32(0), w_before), w_after)


@pytest.mark.parametrize("variant", VARIANTS)
def test_resampling_bit_exact(variant):
    f, p = load(variant)
    P = int(f["P"])
    for fr in steady_frames(f):
        cum = f[f"f{fr}_joint_cum"]
        jmax = cum[-1]
        keys = np.sort(O.resample_keys(p.seed, fr, P))
        u = (jmax * (keys.astype(np.float32) * np.float32(2.0 ** -24))).astype(np.float32)
        anc = O.lower_bound_rule(cum, u)
        srt, bir = particles(f, f"f{fr}_sorted"), particles(f, f"f{fr}_birth")
        nxt = particles(f, f"f{fr}_next")
        pers = anc < P
        for k in ("pos", "vel", "cell", "associated"):
            exp = np.where(pers[:, None] if srt[k].ndim == 2 else pers, srt[k][np.minimum(anc, P - 1)],
                           bir[k][np.maximum(anc - P, 0)])
            np.testing.assert_array_equal(exp, nxt[k], err_msg=f"frame {fr} {k}")
        np.testing.assert_array_equal(nxt["weight"], np.full(P, jmax / np.float32(P), np.float32))


@pytest.mark.parametrize("variant", VARIANTS)
def test_exact_scan_close_to_reference_scan(variant):
    """The oracle's exact prefix differs from thrust's FP32 scan only by FP32 rounding."""
    f, _ = load(variant)
    for fr in steady_frames(f):
        born = f[f"f{fr}_born"]
        ex = O.exact_scan(born)
        np.testing.assert_allclose(ex, f[f"f{fr}_born_cum"], rtol=1e-5, atol=1e-6 * float(ex[-1]))
        exact64 = np.cumsum(born.astype(np.float64))
        np.testing.assert_allclose(ex, exact64, rtol=6e-8, atol=1e-30)


# ------------------------------------------------------------------ DS-PHD/MIB
def test_ds_measurement_grid_matches_reference():
    """calcMeasurementGridKernel restated in FP32: the neighbour sets and every branch agree; the
    values agree to 2 ulp (pOcc uses libm's expf against CUDA's)."""
    f, p = load("dsphdmib")
    G, Gz = int(f["G"]), int(f["Gz"])
    for fr in frames(f):
        o = O.ds_measgrid(G, Gz, p.resolution, f[f"f{fr}_sensor_rel"], p.max_range, p.meas_occ_stddev,
                          f[f"f{fr}_pts"])
        ro, rf = f[f"f{fr}_meas_occ"], f[f"f{fr}_meas_free"]
        ok = o["tie"] == 0
        assert ok.mean() > 0.999
        for mine, ref in ((o["meas_occ"], ro), (o["meas_free"], rf)):
            np.testing.assert_array_equal(mine[ok] <= 1e-5, ref[ok] <= 1e-5)  # same branch
            np.testing.assert_allclose(mine[ok], ref[ok], rtol=2.5e-7, atol=0)
        assert np.array_equal(o["nbr"] > 0, (ro > 0) | (rf > 0))


def ds_update_mirror(meas_occ, meas_free, occ_in, free_in, has, sw32, p_B):
    """src/dsphdmib/kernel/mass_update.cu:12-87 with its float/double promotions."""
    f32, f64 = np.float32, np.float64
    mop = np.where(has, sw32, f32(0)).astype(f32)
    mop = np.where(has & (mop > 1), f32(1), mop).astype(f32)
    m_in = np.where(has, mop, occ_in).astype(f32)
    mfp = np.minimum((f32(0.9) * free_in).astype(f32), (f32(1) - m_in).astype(f32)).astype(f32)
    unknown = (f64(1) - m_in.astype(f64) - mfp.astype(f64)).astype(f32)
    mu = (f64(1) - meas_free.astype(f64) - meas_occ.astype(f64)).astype(f32)
    K = ((mfp * meas_occ).astype(f32) + (m_in * meas_free).astype(f32)).astype(f32)
    no = (((m_in * mu).astype(f32) + (unknown * meas_occ).astype(f32)).astype(f32) + (m_in * meas_occ).astype(f32))
    nf = (((mfp * mu).astype(f32) + (unknown * meas_free).astype(f32)).astype(f32) + (mfp * meas_free).astype(f32))
    den = f64(1) - K.astype(f64)
    occ = (no.astype(f32).astype(f64) / den).astype(f32)
    fr = (nf.astype(f32).astype(f64) / den).astype(f32)
    om = f64(1) - mop.astype(f64)
    born = np.where(has, ((occ * f32(p_B)).astype(f32).astype(f64) * om) / (mop.astype(f64) + f64(f32(p_B)) * om),
                    0.0).astype(f32)
    return occ, fr, born, (occ - born).astype(f32), mop


def test_ds_update_bit_exact_and_fp64():
    f, p = load("dsphdmib")
    C_ = int(f["G"]) ** 2 * int(f["Gz"])
    for fr in steady_frames(f):
        cin = f[f"f{fr}_cells_in"]
        cout = f[f"f{fr}_cells_occ"]
        srt = particles(f, f"f{fr}_sorted")
        sw32 = np.zeros(C_, np.float32)  # the reference's sequential FP32 sum (:60-62)
        for i in range(srt["cell"].size):
            sw32[srt["cell"][i]] += srt["weight"][i]
        has = cin["start_idx"] >= 0
        occ, fr_, born, pers, pred = ds_update_mirror(f[f"f{fr}_meas_occ"], f[f"f{fr}_meas_free"],
                                                      cin["occ_mass"], cin["free_mass"], has, sw32, p.birth_prob)
        np.testing.assert_array_equal(occ, cout["occ_mass"])
        np.testing.assert_array_equal(fr_, cout["free_mass"])
        np.testing.assert_array_equal(born, f[f"f{fr}_born"])
        np.testing.assert_array_equal(pers, cout["pers_mass"])
        np.testing.assert_array_equal(pred, cout["pred_mass"])
        # FP64 oracle: same equations, every mass within 1e-5 on the cell's occupancy scale
        sw, swx, swy, swz = O.cell_sums(srt["cell"], srt["weight"], srt["vel"], C_)
        o = O.ds_update(p.birth_prob, f[f"f{fr}_meas_occ"], f[f"f{fr}_meas_free"], cin["occ_mass"],
                        cin["free_mass"], has.astype(np.int32), sw, swx, swy, swz)
        for name, field in [("occ", "occ_mass"), ("free", "free_mass"), ("pred", "pred_mass")]:
            assert relerr(cout[field], o[name], 1e-4).max() < 1e-5, (fr, name)
        scale = np.maximum(np.abs(o["occ"]), 1e-4)
        assert (np.abs(cout["pers_mass"] - o["pers"]) / scale).max() < 1e-5
        assert (np.abs(f[f"f{fr}_born"] - o["born"]) / scale).max() < 1e-5
        # in-place normalisation (mass_update.cu:37-44,64-68), bit-exact with the FP32 sum
        w = srt["weight"].copy()
        norm = sw32[srt["cell"]] > 1.0
        w[norm] = w[norm] / sw32[srt["cell"]][norm]
        np.testing.assert_array_equal(w, f[f"f{fr}_sorted_after_occ_weight"])


# ------------------------------------------------------------------ ego-motion map shift
def load_shift():
    path = GOLD / "k3dom_shift_small.npz"
    if not path.exists():
        pytest.skip(f"{path.name} not generated")
    f = np.load(path)
    return f, N.Params.from_buffer_copy(f["params"].tobytes())


def test_map_shift_matches_reference():
    """DOM_c::updatePose with ego motion (src/common/dom.cu:111-158): the integer move, the shift
    condition, the new map centre, the shifted 68-byte cells (initGridCellsKernel +
    moveMapKernel) and the shifted particle positions (moveParticlesKernel) of the oracle equal
    the reference's, bit for bit, on every frame of a 0.6 m/frame sequence; frames below the
    threshold leave cells, particles and centre untouched."""
    f, p = load_shift()
    G, Gz = int(f["G"]), int(f["Gz"])
    off = np.array([p.sensor_off_x, p.sensor_off_y, p.sensor_off_z], np.float32)
    n_shift = 0
    moves = []
    for fr in range(1, max(frames(f)) + 1):
        c0, c1 = f[f"f{fr}_center_before"], f[f"f{fr}_center_after"]
        mv = O.map_move(f[f"f{fr}_pose"], c0, off, p.resolution)
        cells0, cells1 = f[f"f{fr}_cells_before"], f[f"f{fr}_cells_after"]
        pos0, pos1 = f[f"f{fr}_pos_before"], f[f"f{fr}_pos_after"]
        if O.map_shift_fires(mv, p.map_shift_thresh):
            n_shift += 1
            moves.append(mv)
            exp_c = (c0 + mv.astype(np.float32) * np.float32(p.resolution)).astype(np.float32)
            np.testing.assert_array_equal(c1, exp_c)
            exp = O.shift_gridcells(cells0, mv, G, Gz, p.prior_free, p.prior_static, p.prior_dynamic, p.prior_occ)
            assert exp.tobytes() == cells1.tobytes(), f"frame {fr}: shifted cells"
            np.testing.assert_array_equal(O.shift_positions(pos0, mv), pos1, err_msg=f"frame {fr}: positions")
        else:
            np.testing.assert_array_equal(c1, c0)
            assert cells0.tobytes() == cells1.tobytes()
            np.testing.assert_array_equal(pos0, pos1)
    assert n_shift >= 2, "the sequence must shift the map at least twice"
    assert any(np.any(m < 0) for m in moves) or any(np.any(m > 0) for m in moves)


def test_prediction_after_shift_bit_exact():
    """The shift folded into prediction: predicting the unshifted set with the pending move
    subtracted first (orc_predict's shift argument, as the library's k_predict does) equals the
    reference's moveParticlesKernel followed by predictKernel."""
    f, p = load_shift()
    G, Gz = int(f["G"]), int(f["Gz"])
    off = np.array([p.sensor_off_x, p.sensor_off_y, p.sensor_off_z], np.float32)
    seen = 0
    for fr in range(1, max(frames(f)) + 1):
        mv = O.map_move(f[f"f{fr}_pose"], f[f"f{fr}_center_before"], off, p.resolution)
        fires = O.map_shift_fires(mv, p.map_shift_thresh)
        st = {"pos": f[f"f{fr}_pos_before"], "vel": f[f"f{fr}_pred_in_vel"], "weight": f[f"f{fr}_pred_in_weight"]}
        out = O.predict(st, f[f"f{fr}_normals"], G, Gz, float(f[f"f{fr}_dt"]), p.persistence_prob,
                        p.stddev_process_noise_position, p.stddev_process_noise_velocity, p.init_max_velocity,
                        shift=tuple(int(v) for v in mv) if fires else None)
        for k in ("pos", "vel", "weight", "cell"):
            np.testing.assert_array_equal(out[k], f[f"f{fr}_pred_out_{k}"], err_msg=f"frame {fr} {k}")
        seen += fires
    assert seen >= 2


def test_mappoint_coordinates_match_reference_formula():
    """index_to_coord restates DOM_c::indexToCoord{X,Y,Z} (include/common/dom.h:70-81); the
    fixture's centres after each shift exercise non-zero map centres."""
    f, p = load_shift()
    G = int(f["G"])
    for fr in range(1, max(frames(f)) + 1):
        idx = f[f"f{fr}_coord_idx"]
        got = O.index_to_coord(idx, G, p.resolution, p.size, p.size_z, f[f"f{fr}_center_after"])
        np.testing.assert_array_equal(got, f[f"f{fr}_coords"])
