"""Parity of the CUDA path (through the C ABI) with the oracle and with the reference's own CUDA.

The library runs stage by stage (the reference's public stage methods) in lockstep with the
reference harness (oracle/_ref, the reference's sources built unmodified) and the CPU oracle.
Before each stage the reference receives the library's state, so each stage is compared on
identical inputs and identical Philox draws.

Bars
  * bit-exact: voxel indices after prediction, the sort permutation and sorted set, cell
    ranges, first-frame and birth slots, birth velocities, ancestors and the resampled set
    (against the oracle, whose exact prefix sums the library reproduces); the map shift of
    cells, map centre and particles;
  * 1e-5 relative (floor 1e-3 of the mass scale): the evidence against the FP64 oracle; masses,
    born, persistent and predicted masses, mean velocities and the reweight factor mu_UA against
    the FP64 update of the library's own evidence; masses end to end against the FP64 oracle,
    with the FP64 update's own change between the two evidence values as the allowance (the
    update moves mass by ~sqrt(evidence), so near zero evidence it is ill-conditioned);
  * against the reference: predictions and the sorted set are bit-exact; every slot and
    ancestor that differs from the reference's lies within the worst-case FP32 rounding bound
    of its thrust prefix sum of a boundary (tie rule; the flips are counted and printed); the
    reweighted weights agree to 2 ulp on identical cells; the reference's masses equal the
    oracle's FP32 restatement of its arithmetic to 1e-5 (its only difference from the library
    is that FP32 arithmetic: free-evidence cancellation, dropped NaN terms).
"""
import numpy as np
import pytest

import k3dom_b200 as K
from k3dom_b200 import scene
from oracle import binding as O

pytestmark = pytest.mark.gpu

RTOL = 1e-5


def rel_ok(got, exp, floor, rtol=RTOL, allow=None):
    got = np.asarray(got, np.float64)
    exp = np.asarray(exp, np.float64)
    err = np.abs(got - exp)
    bound = rtol * np.maximum(np.abs(exp), floor)
    if allow is not None:
        bound = bound + allow
    bad = err > bound
    return bad.sum(), (err / np.maximum(np.abs(exp), floor)).max()


U32 = 2.0 ** -24  # unit roundoff of FP32


def scan_bound_ulps(n):
    """Worst-case FP32 rounding, in units of the unit roundoff times the prefix, of an
    inclusive prefix sum of n non-negative floats whose carry chain takes one addition per tile
    of at least 1,024 elements plus at most 64 additions inside a tile (any CUB/thrust tiling of
    the reference's thrust::inclusive_scan, include/common/common.h:7-18), applied twice (the
    prefix and the total it is normalised by or drawn against), plus the normalising product."""
    h = -(-int(n) // 1024) + 64
    return 2 * h + 4


def check_boundary_flips(got, ref, bounds, targets, bound_rel, what, alt=None):
    """Tie rule for integers decided by an FP32 prefix sum. got[i] is the library's cell/index
    (exact prefix), ref[i] the reference's; where they differ, j = min(got[i], ref[i]) is the
    boundary that decided it, and targets[i] must lie within bound_rel * bounds[j] of
    bounds[j] (the exact boundary). alt(i) may return further accepted boundaries (a stale slot
    the reference left unwritten). Returns the number of flips."""
    diff = np.nonzero(got != ref)[0]
    bad = []
    for i in diff:
        cand = [min(int(got[i]), int(ref[i]))]
        if alt is not None:
            cand += alt(i)
        ok = False
        for j in cand:
            if 0 <= j < bounds.size:
                b = float(bounds[j])
                if abs(b - float(targets[i])) <= bound_rel * abs(b) + 1e-30:
                    ok = True
                    break
        if not ok:
            bad.append(int(i))
    assert not bad, f"{what}: {len(bad)} of {diff.size} differences are not scan-rounding ties, first {bad[:5]}"
    return int(diff.size)


STATE_FIELDS = ("start_idx", "end_idx", "mean_x_vel", "mean_y_vel", "mean_z_vel", "likelihood", "p_A",
                "free_mass", "static_mass", "dynamic_mass", "occ_mass", "pers_mass", "pred_mass")


def small_cfg(variant, **kw):
    sizes = dict(G=32, Gz=8, res=0.2, P=8192, B=2048, n_points=1500)
    sizes.update(kw)
    cfg = scene.small(seed=7, variant=variant, **sizes)
    cfg.params["seed"] = 1234
    return cfg


class Lockstep:
    def __init__(self, cfg, with_reference=True):
        self.cfg = cfg
        self.variant = cfg.variant
        self.p = K.make_params(cfg.variant, **cfg.params)
        self.lib = K.DOM(self.p, cfg.variant)
        self.G, self.Gz, self.C = self.lib.grid_size, self.lib.grid_size_z, self.lib.grid_cell_count
        self.P, self.B = self.lib.particle_count, self.lib.new_born_particle_count
        self.ref = None
        if with_reference and O.reference_available(cfg.variant):
            self.ref = O.Reference(self.p, cfg.variant)
        self.off = np.array([self.p.sensor_off_x, self.p.sensor_off_y, self.p.sensor_off_z], np.float32)
        self.t_prev = None
        self.report = {}
        self.shift_frames = []
        self.empty_frames = set()  # frames whose scan is replaced by zero points

    def scan(self, f, t):
        s, pts = self.cfg.scene.scan(f, t, self.cfg.n_points)
        if f in self.empty_frames:
            pts = np.zeros((0, 3), np.float32)
        return s, pts

    def close(self):
        self.lib.close()
        if self.ref:
            self.ref.close()

    def sensor_rel(self):
        i = self.lib.info()
        return np.array([i.sensor_x - i.center_x, i.sensor_y - i.center_y, i.sensor_z - i.center_z], np.float32)

    def center(self):
        i = self.lib.info()
        return np.array([i.center_x, i.center_y, i.center_z], np.float32)

    def count(self, key, n):
        self.report[key] = self.report.get(key, 0) + int(n)

    # -------------------------------------------------------------- oracle helpers
    def oracle_evidence(self, pts):
        return O.bgki(self.G, self.Gz, self.p.resolution, self.sensor_rel(), self.p.ls, self.p.sigma, pts)

    def check_tie_cells(self, tie, ev_cells):
        """Cells whose evidence holds a tied (cell, point) pair are left out of the mass bars;
        there must be few of them: at most 1e-3 of the cells with evidence (and 16)."""
        n_tie = int((tie != 0).sum())
        self.count("tie_cells", n_tie)
        assert n_tie <= max(16, int(1e-3 * max(int(ev_cells), 1))), ("tie cells", n_tie, int(ev_cells))

    def check_masses_k3dom(self, cells_in, sorted_set, pts, dt, first):
        lib = self.lib
        ev = self.oracle_evidence(pts)
        if first:
            z = np.zeros(self.C)
            has = np.zeros(self.C, np.int32)
            sums = (z, z, z, z)
        else:
            has = (cells_in["start_idx"] >= 0).astype(np.int32)
            sums = O.cell_sums(sorted_set["cell"], sorted_set["weight"], sorted_set["vel"], self.C)
        o = O.k3dom_update(dt, self.p.gamma, self.p.birth_prob, self.p.mass_scale, ev, cells_in["free_mass"],
                           cells_in["static_mass"], cells_in["dynamic_mass"], has, *sums)
        tie = ev["tie_mass"]
        # evidence first: tied pairs may flip a whole term
        got_f = lib.get_cell_field("del_free")
        n, e = rel_ok(got_f, ev["del_free"], 1e-2 * self.p.sigma, allow=tie * 1.0001)
        assert n == 0, ("del_free", n, e)
        n, e = rel_ok(lib.get_cell_field("del_occ"), ev["del_occ"], 1e-2 * self.p.sigma)
        assert n == 0, ("del_occ", n, e)
        self.check_tie_cells(tie, ((ev["del_free"] > 0) | (ev["del_occ"] > 0)).sum())
        ok = tie == 0
        # The mass update (mass_update.cu:106-137) moves mass by credit(sqrt(z))/z * del with
        # z = del * sum of masses, i.e. by ~sqrt(del), and between static and dynamic mass by
        # (del_occ - del_free)+ and (del_free - del_occ)+: near zero evidence, and where the two
        # evidence terms nearly cancel, it turns small evidence differences into larger mass
        # differences; and the prediction splits (free + dynamic) into dynamic = the particles'
        # weight sum and free = the rest, which cancels where the two are close. So the masses are
        # held (a) to the FP64 update applied to the library's own inputs (its evidence, and the
        # per-cell weight sums it stores in FP32 as the reference's GridCell does), 1e-5 plus what
        # the update moves within the FP32 rounding of those inputs (the library updates from the
        # exact evidence sums and rounds each FP64 weight sum once), and (b) end to end to the
        # FP64 oracle, with (a)'s allowance plus what the FP64 update itself moves between the
        # two sets of inputs; the cells that need an allowance are counted.
        ev_lib = {"del_occ": lib.get_cell_field("del_occ").astype(np.float64),
                  "del_free": lib.get_cell_field("del_free").astype(np.float64)}
        sums_lib = tuple(np.asarray(x, np.float32).astype(np.float64) for x in sums)

        def update(e, sw=None):
            s_ = sums_lib if sw is None else (sw,) + sums_lib[1:]
            return O.k3dom_update(dt, self.p.gamma, self.p.birth_prob, self.p.mass_scale, e, cells_in["free_mass"],
                                  cells_in["static_mass"], cells_in["dynamic_mass"], has, *s_)

        def half_ulp(v):
            return np.where(v > 0, 0.5 * np.spacing(np.abs(v).astype(np.float32)).astype(np.float64), 0.0)
        o_lib = update(ev_lib)
        half = {k: half_ulp(v) for k, v in ev_lib.items()}
        hw = half_ulp(sums_lib[0])
        # (evidence and weight sums are never negative: a zero stays zero)
        corners = [update({"del_occ": np.maximum(ev_lib["del_occ"] + so * half["del_occ"], 0.0),
                           "del_free": np.maximum(ev_lib["del_free"] + sf * half["del_free"], 0.0)},
                          np.maximum(sums_lib[0] + sw * hw, 0.0))
                   for so in (-1.0, 1.0) for sf in (-1.0, 1.0) for sw in (-1.0, 1.0)]
        for fld, key in [("free_mass", "free"), ("static_mass", "static"), ("dynamic_mass", "dyn"),
                         ("born_mass", "born"), ("pred_mass", "pred")]:
            got = lib.get_cell_field(fld)
            export = np.max([np.abs(c[key] - o_lib[key]) for c in corners], axis=0)
            assert np.isfinite(export).all(), (fld, "allowance")
            n, e = rel_ok(got[ok], o_lib[key][ok], 1e-3, allow=export[ok])
            if n:
                self.dump_cells(fld, key, got, o_lib, ev, cells_in, sums, has, ok)
            assert n == 0, (fld, "vs FP64 update of the library's evidence", n, e)
            self.count(f"export_conditioned_{fld}",
                       int(((np.abs(got.astype(np.float64) - o_lib[key]) >
                             RTOL * np.maximum(np.abs(o_lib[key]), 1e-3)) & ok).sum()))
            cond = np.abs(o_lib[key] - o[key]) + export
            n, e = rel_ok(got[ok], o[key][ok], 1e-3, allow=cond[ok])
            if n:
                self.dump_cells(fld, key, got, o, ev, cells_in, sums, has, ok)
            assert n == 0, (fld, "vs FP64 oracle", n, e)
            needs = (np.abs(got.astype(np.float64) - o[key]) > RTOL * np.maximum(np.abs(o[key]), 1e-3)) & ok
            self.count(f"ill_conditioned_{fld}", int(needs.sum()))
            self.report[f"max_rel_{fld}"] = max(self.report.get(f"max_rel_{fld}", 0.0), float(e))
        # the quantities derived from the masses, against the FP64 update of the library's evidence
        dscale = np.maximum(np.abs(o_lib["dyn"]), 1e-3)
        pers = lib.get_cell_field("pers_mass")
        export = np.max([np.abs(c["pers"] - o_lib["pers"]) for c in corners], axis=0)
        assert ((np.abs(pers - o_lib["pers"]) - export) / dscale)[ok].max() < RTOL
        self.mu_export = np.max([np.abs(c["mu"] - o_lib["mu"]) for c in corners], axis=0)
        if not first:
            for fld, key in [("mean_x_vel", "mvx"), ("mean_y_vel", "mvy"), ("mean_z_vel", "mvz")]:
                got = lib.get_cell_field(fld)
                # the mean is sum(w v) / pers: relative to the speed scale where pers is tiny
                n, e = rel_ok(got[ok], o_lib[key][ok], 1.0, rtol=RTOL)
                assert n == 0, (fld, n, e)
                self.report["max_rel_mean_vel"] = max(self.report.get("max_rel_mean_vel", 0.0), float(e))
        return o_lib, ev

    def dump_cells(self, fld, key, got, o, ev, cells_in, sums, has, ok):
        """Prints every input and output of the worst cells of a failed mass bar."""
        err = np.abs(got.astype(np.float64) - o[key]) / np.maximum(np.abs(o[key]), 1e-3)
        err[~ok] = 0
        lib = self.lib
        fields = {k: lib.get_cell_field(k) for k in ("free_mass", "static_mass", "dynamic_mass", "born_mass",
                                                     "pred_mass", "pers_mass", "del_occ", "del_free")}
        for c in np.argsort(-err)[:6]:
            print(f"cell {c} err {err[c]:.3g} has {has[c]} in f/s/d {cells_in['free_mass'][c]:.9g} "
                  f"{cells_in['static_mass'][c]:.9g} {cells_in['dynamic_mass'][c]:.9g} start {cells_in['start_idx'][c]}")
            print("   oracle", {k: float(o[k][c]) for k in ("free", "static", "dyn", "born", "pred", "pers")},
                  "sum_w", float(sums[0][c]), "ev", float(ev["del_occ"][c]), float(ev["del_free"][c]),
                  "tie", float(ev["tie_mass"][c]))
            print("   lib   ", {k: float(v[c]) for k, v in fields.items()})

    def check_mu(self, o, ok):
        """The reweight factor mu_UA = pers / pred (update_persistent_particles.cu:17-55) against
        the FP64 oracle; pers carries an error of 1e-5 of the dynamic mass, so mu's bar is that
        over pred where it is larger than 1e-5 of mu."""
        mu = self.lib.get_cell_field("mu_UA").astype(np.float64)
        has = (o["pred"] > 0) & ok
        scale = np.maximum(np.abs(o["mu"]), np.maximum(np.abs(o["dyn"]), 1e-3) / np.where(o["pred"] > 0, o["pred"], 1))
        # less what the update moves within the FP32 rounding of the exported evidence
        export = getattr(self, "mu_export", np.zeros_like(mu))
        err = (np.maximum(np.abs(mu - o["mu"]) - export, 0.0) / scale)[has]
        assert err.size == 0 or err.max() < RTOL, ("mu_UA", float(err.max()))
        self.report["max_rel_mu_UA"] = max(self.report.get("max_rel_mu_UA", 0.0), float(err.max()) if err.size else 0.0)

    def check_ref_masses_k3dom(self, cells_in, sorted_set, pts, dt, first):
        """The reference's own masses after its occupancy update, on the library's input cells,
        sorted particles and points, equal the oracle's FP32 restatement of its arithmetic
        (BGKI mass_update.cu:32-77 and the cell update :79-183 in FP32, serial weight sums)."""
        rc = self.ref.cells()
        dp = np.zeros(self.C, np.float32)
        if not first:
            np.add.at(dp, sorted_set["cell"], sorted_set["weight"])  # in index order, as the serial loop
        ev32 = O.bgki_ref32(self.G, self.Gz, self.p.resolution, self.sensor_rel(), self.p.ls, self.p.sigma, pts)
        m = O.k3dom_update_ref32(dt, self.p.gamma, self.p.birth_prob, self.p.mass_scale, ev32, cells_in["free_mass"],
                                 cells_in["static_mass"], cells_in["dynamic_mass"], dp)
        worst = 0.0
        for name, field in [("free", "free_mass"), ("static", "static_mass"), ("dyn", "dynamic_mass")]:
            e = np.abs(rc[field].astype(np.float64) - m[name]) / np.maximum(np.abs(m[name]), 1e-3)
            assert e.max() < RTOL, ("reference vs FP32 restatement", field, float(e.max()))
            lc = self.lib.get_cell_field(field)
            worst = max(worst, float((np.abs(rc[field] - lc) / np.maximum(np.abs(lc), 1e-3)).max()))
        self.report["ref_vs_lib_mass_max_rel"] = worst  # the reference's FP32 error, reported

    # -------------------------------------------------------------- frames
    def first_frame(self):
        cfg, lib, ref = self.cfg, self.lib, self.ref
        t = 0.1
        s, pts = self.scan(0, t)
        lib.updatePose(*s)
        cells_in = lib.get_gridcells()
        prev_cell = lib.get_particles("persistent")["cell"]
        lib.initializeParticles(pts)
        born = lib.get_cell_field("born_mass")
        if self.variant == "k3dom":
            self.check_masses_k3dom(cells_in, None, pts, 0.0, True)
        else:
            self.check_ds(cells_in, None, pts, first=True)
        # first-frame particles: exact prefix of the library's born masses -> slots
        cum = O.exact_scan(born)
        _, bc, _ = lib.resampling_state()
        np.testing.assert_array_equal(bc, cum)
        o = O.init_particles(cum, self.P, self.G, self.p.init_max_velocity, self.p.particle_min_vel,
                             O.uniforms(self.p.seed, 0, 2, 0, self.P), prev_cell=prev_cell)
        got = lib.get_particles("persistent")
        for k in ("cell", "pos", "vel", "weight"):
            np.testing.assert_array_equal(got[k], o[k], err_msg=f"init {k}")
        if ref is not None:
            ref.update_pose(*s)
            ref.init_particles(0, pts)
            r = ref.particles(0)
            np.testing.assert_array_equal(r["vel"], got["vel"])  # draws are per slot: identical
            # slots: initParticlesKernel1 (init_new_particles.cu:54-68). The reference formed its own
            # born masses (its FP32 evidence), so its slots are held to the slot rule applied to
            # those masses, exactly, with flips only within the FP32 bound of its thrust scan
            ref_cum = O.exact_scan(ref.born())
            o_ref = O.init_particles(ref_cum, self.P, self.G, self.p.init_max_velocity, self.p.particle_min_vel,
                                     O.uniforms(self.p.seed, 0, 2, 0, self.P), prev_cell=prev_cell)
            self.count("init_slot_flips_vs_ref", self.slot_flips(o_ref["cell"], r["cell"], ref_cum, self.P,
                                                                 prev_cell, "first-frame slots"))
            ref.finish(t, False)
        lib.finishFrame(t)
        self.t_prev = t

    def slot_flips(self, got_cell, ref_cell, cum_exact, v, prev_cell, what):
        """Slot i belongs to the first cell j with int(acc[j] * v / acc[-1]) > i
        (init_new_particles.cu:14-27,44-52); a flip must have i + 1 within the scan bound of the
        decisive boundary acc[j] * v / acc[-1]. A slot that either side left unwritten keeps its
        previous cell (the last slots, when the FP32 product acc[-1] * (v / acc[-1]) rounds below
        v): then the decisive boundary is the other side's cell's or the last one."""
        e_n = cum_exact.astype(np.float64) * (float(v) / float(cum_exact[-1]))
        rel = scan_bound_ulps(cum_exact.size) * U32
        targets = np.arange(1, got_cell.size + 1, dtype=np.float64)

        def alt(i):
            if prev_cell is not None and (ref_cell[i] == prev_cell[i] or got_cell[i] == prev_cell[i]):
                return [int(got_cell[i]), int(ref_cell[i]), e_n.size - 1]
            return []
        return check_boundary_flips(got_cell, ref_cell, e_n, targets, rel, what, alt)

    def steady_frame(self, f):
        cfg, lib, ref, p = self.cfg, self.lib, self.ref, self.p
        t = 0.1 + f * cfg.dt
        dt = float(np.float32(t) - np.float32(self.t_prev))
        s, pts = self.scan(f, t)
        # ---- pose: the map shift (src/common/dom.cu:111-158) against the oracle's restatement
        cells_pre, center_pre = lib.get_gridcells(), self.center()
        lib.updatePose(*s)
        mv = O.map_move(s, center_pre, self.off, p.resolution)
        shift = O.map_shift_fires(mv, p.map_shift_thresh)
        if shift:
            self.shift_frames.append(f)
            exp = O.shift_gridcells(cells_pre, mv, self.G, self.Gz, p.prior_free, p.prior_static, p.prior_dynamic,
                                    p.prior_occ)
            got = lib.get_gridcells()
            for fld in STATE_FIELDS:
                np.testing.assert_array_equal(got[fld], exp[fld], err_msg=f"map shift {fld}")
            np.testing.assert_array_equal(self.center(),
                                          (center_pre + mv.astype(np.float32) * np.float32(p.resolution)))
        else:
            np.testing.assert_array_equal(self.center(), center_pre)
        if ref is not None:
            ref.update_pose(*s)
            np.testing.assert_array_equal(ref.center(), self.center())
        # ---- prediction (the pending shift is folded into the library's prediction)
        a = lib.get_particles("persistent")
        if ref is not None:
            a_ref = dict(a)
            if shift:
                a_ref["pos"] = O.shift_positions(a["pos"], mv)
            ref.set_particles(0, **a_ref)
        lib.particlePrediction(dt)
        got = lib.get_particles("persistent")
        normals = K.debug_draws(p.seed, f, 1, 0, self.P)
        o = O.predict(a, normals, self.G, self.Gz, dt, p.persistence_prob, p.stddev_process_noise_position,
                      p.stddev_process_noise_velocity, p.init_max_velocity,
                      shift=tuple(int(v) for v in mv) if shift else None)
        for k in ("pos", "vel", "weight", "cell"):
            np.testing.assert_array_equal(got[k], o[k], err_msg=f"predict {k}")
        if ref is not None:
            ref.predict(f, dt)
            r = ref.particles(0)
            for k in ("pos", "vel", "weight", "cell"):
                np.testing.assert_array_equal(got[k], r[k], err_msg=f"predict vs reference {k}")
        # ---- assignment
        lib.particleAssignment()
        perm = lib.sort_permutation()
        operm, osk, ost, oen = O.assign(got["cell"], self.C)
        np.testing.assert_array_equal(perm, operm)
        srt = lib.get_particles("sorted")
        for k in ("pos", "vel", "weight", "cell"):
            np.testing.assert_array_equal(srt[k], got[k][perm], err_msg=f"sorted {k}")
        st, en = lib.get_cell_ranges()
        np.testing.assert_array_equal(st, ost)
        np.testing.assert_array_equal(en, oen)
        self.last_ranges = (st, en)
        if ref is not None:
            ref.assign()
            r = ref.particles(0)
            for k in ("pos", "vel", "weight", "cell", "associated"):
                np.testing.assert_array_equal(srt[k], r[k], err_msg=f"sorted vs reference {k}")
        # ---- occupancy update
        cells_in = lib.get_gridcells()
        if ref is not None:
            ref.set_cells(cells_in)
        lib.gridCellOccupancyUpdate(dt, pts)
        o_mass = None
        if self.variant == "k3dom":
            o_mass, ev = self.check_masses_k3dom(cells_in, srt, pts, dt, False)
        else:
            o_ds = self.check_ds(cells_in, srt, pts, first=False)
        if ref is not None:
            ref.occupancy(dt, pts)
            if self.variant == "k3dom":
                self.check_ref_masses_k3dom(cells_in, srt, pts, dt, False)
        # ---- persistent particles
        self.ref_sorted_weight_before_reweight = srt["weight"]
        lib.updatePersistentParticles()
        mu = lib.get_cell_field("mu_UA")
        w2 = lib.get_particles("sorted")["weight"]
        base = srt["weight"]
        if self.variant == "k3dom":
            np.testing.assert_array_equal(w2, (mu[srt["cell"]] * base).astype(np.float32))
            self.check_mu(o_mass, ev["tie_mass"] == 0)
        else:
            # DS: w' = mu_UA * w / occ_pred where the cell's weights summed above 1
            # (dsphdmib/kernel/mass_update.cu:52-60, update_persistent_particles.cu:49-55)
            c = srt["cell"]
            d = o_ds["div"][c]
            wd = np.abs(base.astype(np.float64)) / np.where(d > 0, d, 1.0)
            exp = o_ds["mu"][c] * wd
            # mu = pers / pred carries pers's error on the occupied-mass scale (the bar of check_ds)
            pred = np.where(o_ds["pred"][c] > 0, o_ds["pred"][c], 1.0)
            mscale = np.maximum(np.abs(o_ds["mu"][c]), np.maximum(np.abs(o_ds["occ"][c]), 1e-4) / pred)
            scale = np.maximum(wd * mscale, 1e-30)
            err = np.abs(np.abs(w2.astype(np.float64)) - exp) / scale
            assert err.max() < RTOL, ("DS reweight", float(err.max()))
            self.count("ds_divided_cells", int((o_ds["div"] > 0).sum()))
        if ref is not None and self.variant == "k3dom":
            # identical cells: the reference reweights with pers / pred of the library's cells
            ref.set_cells(lib.get_gridcells())
            ref.persistent()
            rw = ref.particles(0)["weight"]
            scale = np.maximum(np.abs(w2.astype(np.float64)), np.finfo(np.float32).tiny)
            ulp2 = 2.0 * 2.0 ** -23
            bad = np.abs(rw.astype(np.float64) - w2) > ulp2 * scale
            assert not bad.any(), ("reweight vs reference", int(bad.sum()))
        elif ref is not None:
            ref.persistent()
        # ---- births
        born = lib.get_cell_field("born_mass")
        prev_b = lib.get_particles("birth")
        lib.initializeNewParticles()
        cum = O.exact_scan(born)
        ob = O.births(born, cum, self.B, self.G, 0.0, p.init_max_velocity, p.particle_min_vel,
                      O.uniforms(p.seed, f, 3, 0, self.B), prev_cell=prev_b["cell"],
                      prev_assoc=prev_b["associated"])
        gb = lib.get_particles("birth")
        for k in ("cell", "associated", "pos", "vel", "weight"):
            np.testing.assert_array_equal(gb[k], ob[k], err_msg=f"births {k}")
        if ref is not None:
            ref.set_born(born)
            ref.set_particles(2, cell=prev_b["cell"], associated=prev_b["associated"])
            ref.births(f)
            rb = ref.particles(2)
            np.testing.assert_array_equal(gb["vel"], rb["vel"])
            self.count("birth_slot_flips_vs_ref", self.slot_flips(gb["cell"], rb["cell"], cum, self.B, prev_b["cell"],
                                                                  "birth slots"))
            if self.variant == "k3dom":
                ref.moments()  # statisticalMoments follows the births (src/k3dom/dom.cu:38-41)
                self.check_gridcell_export(gb, rb, prev_b)
        # ---- resampling
        srt2 = lib.get_particles("sorted")
        v = srt2["vel"]
        m2 = np.float32(p.particle_min_vel) * np.float32(p.particle_min_vel)
        slow = ((v[:, 0] * v[:, 0] + v[:, 1] * v[:, 1]) + v[:, 2] * v[:, 2]) < m2
        w_pen = np.where(slow, np.float32(0), srt2["weight"]).astype(np.float32)
        w_b = np.where(ob["slow"] > 0, np.float32(0), gb["weight"]).astype(np.float32)
        if ref is not None:
            ref.set_particles(0, pos=srt2["pos"], vel=srt2["vel"], weight=srt2["weight"], cell=srt2["cell"],
                              associated=srt2["associated"])
            ref.set_particles(2, **gb)
        lib.resampling()
        anc = lib.ancestors()
        oanc, ocum, jmax = O.resample(w_pen, w_b, p.seed, f)
        jc, _, jm = lib.resampling_state()
        np.testing.assert_array_equal(jc, ocum)
        assert jm == jmax
        np.testing.assert_array_equal(anc, oanc)
        nxt = lib.get_particles("persistent")
        pers = anc < self.P
        for k in ("pos", "vel", "cell", "associated"):
            src_p, src_b = srt2[k], gb[k]
            exp = np.where(pers[:, None] if src_p.ndim == 2 else pers, src_p[np.minimum(anc, self.P - 1)],
                           src_b[np.maximum(anc - self.P, 0)])
            np.testing.assert_array_equal(nxt[k], exp, err_msg=f"resampled {k}")
        assert np.all(nxt["weight"] == np.float32(jmax) / np.float32(self.P))
        if ref is not None:
            ref.resampling(f)
            rn = ref.particles(1)
            self.count("ancestor_flips_vs_ref", self.ancestor_flips(rn, srt2, gb, anc, ocum, jmax, f))
            ref.finish(t, True)
        lib.finishFrame(t)
        self.t_prev = t

    def check_gridcell_export(self, gb, rb, prev_b):
        """k3dom_get_gridcell_aos against the reference's own 68-byte GridCell array
        (include/common/dom_types.h:12-45) after the same frame: the reference holds the
        library's cells and recomputed mu_A, mu_UA (update_persistent_particles.cu:17-55), w_A,
        w_UA (init_new_particles.cu:106-121) and the mean velocities
        (statistical_moments.cu:12-63) itself. State fields are bit-exact; mu_UA within 1 ulp
        (FP32 pers / pred against the library's FP64 quotient); mu_A and the mean velocities
        within the FP32 error of the reference's prefix differences (common.h:20-28); w_UA
        bit-exact wherever the two sides gave a cell the same number of birth slots. Then the
        MapPoint export against the node's publish_mapdata formula (k3dom_node.cpp:161-184)
        on these cells, and its coordinates against the reference's indexToCoord."""
        lc, rc = self.lib.get_gridcells(), self.ref.cells()
        for fld in STATE_FIELDS:
            if fld in ("mean_x_vel", "mean_y_vel", "mean_z_vel"):
                continue
            np.testing.assert_array_equal(lc[fld], rc[fld], err_msg=f"GridCell {fld}")
        has = lc["start_idx"] >= 0
        pers = lc["pers_mass"].astype(np.float64)
        pred = lc["pred_mass"].astype(np.float64)
        live = has & (pred > 0)
        mu_l, mu_r = lc["mu_UA"].astype(np.float64), rc["mu_UA"].astype(np.float64)
        assert np.all(np.abs(mu_l - mu_r)[live] <= 2.0 ** -23 * np.abs(mu_l)[live] + 1e-38), "GridCell mu_UA"
        # prefix-difference error of the reference's FP32 scans over the sorted set
        srt = self.lib.get_particles("sorted")  # reweighted sorted set
        st, en = lc["start_idx"], lc["end_idx"]
        rel = scan_bound_ulps(self.P) * U32
        w0 = self.ref_sorted_weight_before_reweight
        cw = np.cumsum(np.abs(w0.astype(np.float64)))
        lo = np.where(st > 0, cw[np.maximum(st - 1, 0)], 0.0)
        hi = cw[np.maximum(en, 0)]
        sum_w = np.where(has, hi - lo, 1.0)
        slack_w = rel * (hi + lo) / np.where(sum_w > 0, sum_w, 1.0)
        mua_l, mua_r = lc["mu_A"].astype(np.float64), rc["mu_A"].astype(np.float64)
        ok = ~live | (np.abs(mua_l - mua_r) <= (slack_w + 2e-6) * np.abs(mua_l) + 1e-30)
        assert ok.all(), ("GridCell mu_A", int((~ok).sum()))
        w2 = srt["weight"].astype(np.float64)
        for k, fld in enumerate(("mean_x_vel", "mean_y_vel", "mean_z_vel")):
            cv = np.cumsum(np.abs(w2 * srt["vel"][:, k]))
            lo_v = np.where(st > 0, cv[np.maximum(st - 1, 0)], 0.0)
            hi_v = cv[np.maximum(en, 0)]
            slack = rel * (hi_v + lo_v) / np.where(pers > 0, pers, 1.0)
            a, b = lc[fld].astype(np.float64), rc[fld].astype(np.float64)
            ok = ~(has & (pers > 0)) | (np.abs(a - b) <= slack + RTOL * np.maximum(np.abs(a), 1.0))
            assert ok.all(), (f"GridCell {fld}", int((~ok).sum()))
        n_l = np.bincount(gb["cell"], minlength=self.C)
        n_r = np.bincount(rb["cell"], minlength=self.C)
        same_n = (n_l == n_r) & (n_l > 0)
        np.testing.assert_array_equal(lc["w_UA"][same_n], rc["w_UA"][same_n], err_msg="GridCell w_UA")
        np.testing.assert_array_equal(lc["w_A"], np.zeros(self.C, np.float32))  # p_A = 0
        self.count("w_UA_count_mismatch_cells", int(((n_l != n_r) & ((n_l > 0) | (n_r > 0))).sum()))
        # MapPoint export
        i = self.lib.info()
        center = np.array([i.center_x, i.center_y, i.center_z], np.float32)
        mp = self.lib.get_mappoints()
        exp = O.mappoints(lc, self.G, self.p.resolution, self.p.size, self.p.size_z, center)
        got = np.stack([mp[n] for n in mp.dtype.names], 1)
        np.testing.assert_array_equal(got, exp)
        idx = np.arange(self.C, dtype=np.int32)
        np.testing.assert_array_equal(got[:, :3], self.ref.index_to_coord(idx))

    def ancestor_flips(self, rn, srt2, gb, anc, cum_exact, jmax, f):
        """calc_resampled_indices (resampling.cu:55-68): ancestor k = lower_bound(acc, u_k) on the
        reference's FP32 scan. Where the reference's resampled particle is not the library's
        ancestor, it must be a nearby joint particle a' and the draw u_k must lie within the
        scan bound of the exact boundary acc[min(a, a')]."""
        P = self.P
        jpos = np.concatenate([srt2["pos"], gb["pos"]])
        jvel = np.concatenate([srt2["vel"], gb["vel"]])
        same = np.all(rn["pos"] == jpos[anc], axis=1) & np.all(rn["vel"] == jvel[anc], axis=1)
        keys = np.sort(O.resample_keys(self.p.seed, f, P))
        u = (np.float32(jmax) * (keys.astype(np.float32) * np.float32(2.0 ** -24))).astype(np.float64)
        ref_anc = anc.copy()
        for k in np.nonzero(~same)[0]:
            found = -1
            for d in range(1, 65):
                for a2 in (int(anc[k]) - d, int(anc[k]) + d):
                    if 0 <= a2 < jpos.shape[0] and np.all(jpos[a2] == rn["pos"][k]) and np.all(jvel[a2] == rn["vel"][k]):
                        found = a2
                        break
                if found >= 0:
                    break
            assert found >= 0, f"resampled particle {k} of the reference is no joint particle near ancestor {anc[k]}"
            ref_anc[k] = found
        rel = scan_bound_ulps(cum_exact.size) * U32
        return check_boundary_flips(anc, ref_anc, cum_exact.astype(np.float64), u, rel, "ancestors")

    # -------------------------------------------------------------- DS
    def check_ds(self, cells_in, sorted_set, pts, first):
        lib, p = self.lib, self.p
        o = O.ds_measgrid(self.G, self.Gz, p.resolution, self.sensor_rel(), p.max_range, p.meas_occ_stddev, pts)
        ok = o["tie"] == 0
        self.check_tie_cells(o["tie"], (o["nbr"] > 0).sum())
        mo, mf = lib.get_cell_field("meas_occ"), lib.get_cell_field("meas_free")
        for mine, exp in ((mo, o["meas_occ"]), (mf, o["meas_free"])):
            np.testing.assert_array_equal(mine[ok] <= 1e-5, exp[ok] <= 1e-5)
            np.testing.assert_allclose(mine[ok], exp[ok], rtol=2.5e-7, atol=0)
        if first:
            np.testing.assert_array_equal(lib.get_cell_field("born_mass"), mo)
            return None
        has = (cells_in["start_idx"] >= 0).astype(np.int32)
        sums = O.cell_sums(sorted_set["cell"], sorted_set["weight"], sorted_set["vel"], self.C)
        u = O.ds_update(p.birth_prob, mo, mf, cells_in["occ_mass"], cells_in["free_mass"], has, *sums)
        for fld, key in [("occ_mass", "occ"), ("free_mass", "free"), ("pred_mass", "pred")]:
            n, e = rel_ok(lib.get_cell_field(fld), u[key], 1e-4)
            assert n == 0, (fld, n, e)
        scale = np.maximum(np.abs(u["occ"]), 1e-4)
        for fld, key in [("pers_mass", "pers"), ("born_mass", "born")]:
            assert (np.abs(lib.get_cell_field(fld) - u[key]) / scale).max() < RTOL, fld
        for fld, key in [("mean_x_vel", "mvx"), ("mean_y_vel", "mvy"), ("mean_z_vel", "mvz")]:
            n, e = rel_ok(lib.get_cell_field(fld), u[key], 1.0, rtol=RTOL)
            assert n == 0, (fld, n, e)
            self.report["max_rel_mean_vel"] = max(self.report.get("max_rel_mean_vel", 0.0), float(e))
        # the reweight factor pers / pred of the DS update (mass_update.cu:12-87 with
        # update_persistent_particles.cu:17-55), against the FP64 oracle on the occupied scale
        mu = lib.get_cell_field("mu_UA").astype(np.float64)
        live = (u["pred"] > 0) & (cells_in["start_idx"] >= 0)
        mscale = np.maximum(np.abs(u["mu"]), np.maximum(np.abs(u["occ"]), 1e-4) / np.where(u["pred"] > 0, u["pred"], 1))
        err = (np.abs(mu - u["mu"]) / mscale)[live]
        assert err.size == 0 or err.max() < RTOL, ("mu_UA", float(err.max()))
        return u


@pytest.mark.parametrize("variant", ["k3dom", "dsphdmib"])
def test_lockstep_small(variant):
    ls = Lockstep(small_cfg(variant))
    try:
        ls.first_frame()
        for f in (1, 2, 3):
            ls.steady_frame(f)
        print(variant, ls.report)
    finally:
        ls.close()


@pytest.mark.parametrize("variant", ["k3dom", "dsphdmib"])
def test_lockstep_config0_scale(variant):
    """Config-0 sizes (64x64x16, P=262144, B=65536, 30000 points) against the oracle."""
    c = scene.config0()
    if variant == "dsphdmib":
        c.params.update(particle_min_vel=0.0, prior_free=0.0, prior_static=0.0, prior_dynamic=0.0)
        c.variant = "dsphdmib"
    c.params["seed"] = 99
    ls = Lockstep(c, with_reference=False)
    try:
        ls.first_frame()
        ls.steady_frame(1)
        print(variant, ls.report)
    finally:
        ls.close()


def test_lockstep_config1_with_map_shift():
    """config1 at full size (256x256x32 voxels: 21-bit cell keys, so the particle sort runs its
    11- and 10-bit radix passes; P=4,194,304, B=1,048,576, 120,000-point scans) with the sensor
    moving at 2.7 m/s: the first frame plus six steady frames, the map shifting (1 m threshold,
    by 11 voxels in x) at frame 5. Every steady frame against the oracle: the shift of cells, centre and particles,
    prediction, the sort permutation, sorted set and cell ranges, birth slots and the resampled
    set bit for bit; masses, born, persistent and predicted masses, mean velocities and mu_UA
    within 1e-5 of FP64."""
    cfg = scene.config1(seed=11)
    cfg.scene.ego_vel = np.array([2.3, -1.4, 0.0])
    cfg.params["seed"] = 2024
    run = Lockstep(cfg, with_reference=False)
    try:
        assert run.C == 2_097_152 and run.P == 4_194_304 and run.B == 1_048_576
        run.first_frame()
        for f in range(1, 7):
            run.steady_frame(f)
        print("config1", run.report, "shift frames", run.shift_frames)
        assert run.shift_frames == [5]
    finally:
        run.close()


def test_lockstep_crowded_cells():
    """Cells holding thousands of particles: their sums span many 128-slot ranges of the sorted
    set (range pieces combined by the fix-up pass), and ranges that lie wholly inside one cell or
    end exactly at a cell boundary. The steady frame checks the sorted set and cell ranges bit for
    bit and the masses built from the sums against the oracle."""
    cfg = small_cfg("k3dom")
    run = Lockstep(cfg, with_reference=False)
    try:
        run.first_frame()
        a = run.lib.get_particles("persistent")
        G = run.G
        rng = np.random.default_rng(3)
        pos, vel, cell = a["pos"].copy(), a["vel"].copy(), a["cell"].copy()
        i = 0
        for n, (x, y, z) in [(5000, (10, 12, 3)), (1500, (20, 8, 4)), (600, (5, 25, 2)), (257, (14, 14, 1)),
                             (256, (15, 14, 1)), (255, (16, 14, 1))]:
            pos[i:i + n] = np.float32([x, y, z]) + rng.uniform(0.3, 0.7, (n, 3)).astype(np.float32)
            cell[i:i + n] = x + G * y + G * G * z
            i += n
        vel[:i] = 0.0
        run.lib.set_particles("persistent", pos=pos, vel=vel, cell=cell)
        run.steady_frame(1)
        st, en = run.last_ranges
        counts = np.where(st >= 0, en - st + 1, 0)
        assert counts.max() >= 4000 and (counts > 256).sum() >= 3
    finally:
        run.close()


def finite_state(lib):
    """Every exported cell field and particle set is free of NaN and infinities."""
    for fld in ("free_mass", "static_mass", "dynamic_mass", "occ_mass", "pers_mass", "pred_mass", "born_mass",
                "mean_x_vel", "mean_y_vel", "mean_z_vel", "mu_UA", "w_UA"):
        assert np.all(np.isfinite(lib.get_cell_field(fld))), fld
    for which in ("persistent", "sorted", "birth"):
        pset = lib.get_particles(which)
        for k in ("pos", "vel", "weight"):
            assert np.all(np.isfinite(pset[k])), (which, k)


@pytest.mark.parametrize("variant", ["k3dom", "dsphdmib"])
def test_degenerate_zero_point_frame(variant):
    """A steady frame without points (the reference loops over zero measurements): status OK,
    every stage against the oracle as in any frame (no evidence: prediction and the mass
    decay only), no NaN, and the next frame with points is exact again."""
    cfg = small_cfg(variant)
    run = Lockstep(cfg, with_reference=False)
    run.empty_frames = {2}
    try:
        run.first_frame()
        for f in (1, 2, 3):
            run.steady_frame(f)
            finite_state(run.lib)
    finally:
        run.close()


def test_degenerate_all_weights_zero_and_no_born_mass():
    """Zero priors and no points on any frame: no cell ever holds mass, so the born masses sum to
    0 (the reference divides by that sum, init_new_particles.cu:44-52: the slot bounds
    int(0 * inf) are 0, no cell owns a slot, the slots keep their cells with weight 0) and every
    joint weight is 0 (joint_max = 0, resampling.cu:55-68: every draw is 0, every ancestor is
    the first particle, weight 0). The library, the oracle and these rules agree bit for bit,
    with status OK and no NaN."""
    cfg = small_cfg("k3dom")
    cfg.params.update(prior_free=0.0, prior_static=0.0, prior_dynamic=0.0, prior_occ=0.0)
    run = Lockstep(cfg, with_reference=False)
    run.empty_frames = {0, 1, 2}
    try:
        run.first_frame()
        assert float(run.lib.get_cell_field("born_mass").sum()) == 0.0
        for f in (1, 2):
            run.steady_frame(f)
            finite_state(run.lib)
            _, born_cum, jmax = run.lib.resampling_state()
            assert jmax == 0.0 and float(born_cum[-1]) == 0.0
            assert np.all(run.lib.ancestors() == 0)
            assert np.all(run.lib.get_particles("persistent")["weight"] == 0.0)
    finally:
        run.close()


def test_degenerate_ds_cell_weight_sum_above_one():
    """DS-PHD/MIB cells whose particle weights sum above 1 (dsphdmib/kernel/mass_update.cu:52-60
    divides every weight in the cell by the sum in place and predicts occupancy 1): crowded
    cells of heavy particles, checked against the oracle's Dempster update and reweight."""
    cfg = small_cfg("dsphdmib")
    run = Lockstep(cfg, with_reference=False)
    try:
        run.first_frame()
        a = run.lib.get_particles("persistent")
        G = run.G
        rng = np.random.default_rng(4)
        pos, vel, w, cell = a["pos"].copy(), a["vel"].copy(), a["weight"].copy(), a["cell"].copy()
        i = 0
        for n, (x, y, z) in [(400, (10, 12, 3)), (300, (20, 8, 4)), (120, (5, 25, 2))]:
            pos[i:i + n] = np.float32([x, y, z]) + rng.uniform(0.3, 0.7, (n, 3)).astype(np.float32)
            vel[i:i + n] = rng.uniform(-0.2, 0.2, (n, 3)).astype(np.float32)
            w[i:i + n] = np.float32(0.01)
            cell[i:i + n] = x + G * y + G * G * z
            i += n
        run.lib.set_particles("persistent", pos=pos, vel=vel, weight=w, cell=cell)
        run.steady_frame(1)
        assert run.report.get("ds_divided_cells", 0) >= 3
        finite_state(run.lib)
    finally:
        run.close()


def test_config1_scale_tilings_agree_and_evidence_matches_oracle():
    """config1 at full size (256 x 256 x 32 voxels, 4,194,304 particles, 120,000-point scans with
    ego motion): three evidence tilings, with 512-, 1024- and 256-ray work items (the last in the
    128-thread build), give bit-identical frames (the evidence is exact fixed point), and the last
    frame's BGKI evidence matches the FP64 oracle within 1e-5 relative (the lockstep bar, ties
    allowed as there)."""
    cfg = scene.config1(seed=7)
    p = K.make_params("k3dom", **cfg.params)
    fields = ["free_mass", "static_mass", "dynamic_mass", "pers_mass", "born_mass", "mean_x_vel", "del_occ",
              "del_free"]
    doms = [K.DOM(p, "k3dom"), K.DOM(p, "k3dom"), K.DOM(p, "k3dom")]
    try:
        pts = None
        for f in range(3):
            t = 0.1 + f * cfg.dt
            s, pts = cfg.scene.scan(f, t, cfg.n_points)
            for d in doms:
                d.updatePose(*s)
                d.updateGrid(t, pts)
            if f == 0:
                doms[0].set_tuning(2, 512)   # 16x16x4 tiles, 512 rays per work item
                doms[1].set_tuning(3, 1024)  # 16x16x8 tiles, 1024 rays per work item
                doms[2].set_tuning(1, 256)   # 8x8x4 tiles, 256 rays per work item
        a = doms[0]
        for b in doms[1:]:
            for fld in fields:
                assert np.array_equal(a.get_cell_field(fld), b.get_cell_field(fld), equal_nan=True), fld
        i = a.info()
        sensor_rel = np.array([i.sensor_x - i.center_x, i.sensor_y - i.center_y, i.sensor_z - i.center_z],
                              np.float32)
        ev = O.bgki(a.grid_size, a.grid_size_z, p.resolution, sensor_rel, p.ls, p.sigma, pts)
        assert (ev["del_free"] > 0).sum() > 100000 and (ev["del_occ"] > 0).sum() > 10000
        n, e = rel_ok(a.get_cell_field("del_free"), ev["del_free"], 1e-2 * p.sigma, allow=ev["tie_mass"] * 1.0001)
        assert n == 0, ("del_free", n, e)
        n, e = rel_ok(a.get_cell_field("del_occ"), ev["del_occ"], 1e-2 * p.sigma)
        assert n == 0, ("del_occ", n, e)
    finally:
        for d in doms:
            d.close()


def test_config1_scale_ds_tilings_agree_and_measurement_matches_oracle():
    """The DS-PHD/MIB variant at config1's full size: two evidence tilings (and rays per work
    item, which changes how the first-100 rule is split across chunks) give bit-identical frames,
    and the last frame's measurement grid matches the oracle's FP32 neighbour sets (the lockstep
    bars; cells whose pOcc comparisons are within 4 ulp of flipping are left out)."""
    cfg = scene.config1(seed=7, variant="dsphdmib")
    p = K.make_params("dsphdmib", **cfg.params)
    fields = ["occ_mass", "free_mass", "pers_mass", "born_mass", "mean_x_vel", "meas_occ", "meas_free"]
    doms = [K.DOM(p, "dsphdmib"), K.DOM(p, "dsphdmib")]
    try:
        pts = None
        for f in range(3):
            t = 0.1 + f * cfg.dt
            s, pts = cfg.scene.scan(f, t, cfg.n_points)
            for d in doms:
                d.updatePose(*s)
                d.updateGrid(t, pts)
            if f == 0:
                doms[0].set_tuning(2, 1024)
                doms[1].set_tuning(1, 256)
        a, b = doms
        for fld in fields:
            assert np.array_equal(a.get_cell_field(fld), b.get_cell_field(fld), equal_nan=True), fld
        i = a.info()
        sensor_rel = np.array([i.sensor_x - i.center_x, i.sensor_y - i.center_y, i.sensor_z - i.center_z],
                              np.float32)
        o = O.ds_measgrid(a.grid_size, a.grid_size_z, p.resolution, sensor_rel, p.max_range, p.meas_occ_stddev, pts)
        ok = o["tie"] == 0
        assert (o["meas_free"][ok] > 1e-5).sum() > 100000
        mo, mf = a.get_cell_field("meas_occ"), a.get_cell_field("meas_free")
        for mine, exp in ((mo, o["meas_occ"]), (mf, o["meas_free"])):
            np.testing.assert_array_equal(mine[ok] <= 1e-5, exp[ok] <= 1e-5)
            np.testing.assert_allclose(mine[ok], exp[ok], rtol=2.5e-7, atol=0)
    finally:
        for d in doms:
            d.close()


def test_draws_equal_oracle():
    for stage in (2, 3, 4):
        for frame in (0, 5):
            a = K.debug_draws(42, frame, stage, 1000, 4096)
            b = O.uniforms(42, frame, stage, 1000, 4096)
            np.testing.assert_array_equal(a, b)
    n = K.debug_draws(42, 3, 1, 0, 4096)
    ref = np.empty(n.size, np.float32)
    O.oracle().orc_normals_libm(42, 3, 0, 4096, ref)
    np.testing.assert_allclose(n.reshape(-1), ref, rtol=2e-6, atol=2e-6)
