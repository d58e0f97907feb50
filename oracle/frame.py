"""TEST INFRASTRUCTURE ONLY: whole frames of the CPU oracle (the reference's updateGrid,
src/k3dom/dom.cu:29-50 and src/dsphdmib/dom.cu:32-53, restated on the CPU).

Used as the CPU baseline of bench.py (the reference itself has no CPU implementation) and by
multi-frame tests. Prediction normals come from libm (not bit-equal to the GPU's); every other
draw is the exact Philox stream.
"""
from __future__ import annotations

import numpy as np

from . import binding as O


class OracleDOM:
    def __init__(self, params, variant="k3dom"):
        p = params
        self.p = p
        self.variant = variant
        self.G = int(np.float32(p.size) / np.float32(p.resolution))
        self.Gz = int(np.float32(p.size_z) / np.float32(p.resolution))
        self.C = self.G * self.G * self.Gz
        self.P, self.B = int(p.particle_count), int(p.new_born_particle_count)
        C_, P, B = self.C, self.P, self.B
        self.free = np.full(C_, p.prior_free, np.float32)
        self.static = np.full(C_, p.prior_static, np.float32)
        self.dyn = np.full(C_, p.prior_dynamic, np.float32)
        self.occ = np.full(C_, p.prior_occ, np.float32)
        self.a = {"pos": np.zeros((P, 3), np.float32), "vel": np.zeros((P, 3), np.float32),
                  "weight": np.zeros(P, np.float32), "cell": np.zeros(P, np.int32),
                  "associated": np.zeros(P, np.uint8)}
        self.birth_cell = np.zeros(B, np.int32)
        self.birth_assoc = np.zeros(B, np.uint8)
        self.first_pose = False
        self.sensor = np.zeros(3, np.float32)
        self.center = np.zeros(3, np.float32)
        self.updated_time = -1.0
        self.frame = 0

    def update_pose(self, x, y, z):
        # DOM_c::updatePose (src/common/dom.cu:111-158); map shift in numpy
        p = self.p
        self.sensor = np.array([x, y, z], np.float32)
        off = np.array([p.sensor_off_x, p.sensor_off_y, p.sensor_off_z], np.float32)
        if not self.first_pose:
            self.first_pose = True
            self.center = (self.sensor - off).astype(np.float32)
            return
        mv = ((self.sensor - self.center - off) / np.float32(p.resolution)).astype(np.float32).astype(np.int64)
        if np.any(np.abs(mv) >= p.map_shift_thresh):
            G, Gz = self.G, self.Gz
            idx = np.arange(self.C)
            x_, y_, z_ = idx % G, (idx % (G * G)) // G, idx // (G * G)
            nx, ny, nz = x_ + mv[0], y_ + mv[1], z_ + mv[2]
            ok = (nx >= 0) & (nx < G) & (ny >= 0) & (ny < G) & (nz >= 0) & (nz < Gz)
            src = np.where(ok, nx + G * ny + G * G * nz, 0)
            for name, prior in (("free", p.prior_free), ("static", p.prior_static), ("dyn", p.prior_dynamic),
                                ("occ", p.prior_occ)):
                arr = getattr(self, name)
                setattr(self, name, np.where(ok, arr[src], np.float32(prior)).astype(np.float32))
            self.a["pos"] = (self.a["pos"] - mv.astype(np.float32)).astype(np.float32)
            self.center = (self.center + mv.astype(np.float32) * np.float32(p.resolution)).astype(np.float32)

    def sensor_rel(self):
        return (self.sensor - self.center).astype(np.float32)

    def _evidence_and_update(self, pts, dt, sorted_set, has):
        p = self.p
        C_ = self.C
        if self.variant == "k3dom":
            ev = O.bgki(self.G, self.Gz, p.resolution, self.sensor_rel(), p.ls, p.sigma, pts)
            if sorted_set is None:
                z = np.zeros(C_)
                sums = (z, z, z, z)
            else:
                sums = O.cell_sums(sorted_set["cell"], sorted_set["weight"], sorted_set["vel"], C_)
            o = O.k3dom_update(dt, p.gamma, p.birth_prob, p.mass_scale, ev, self.free, self.static, self.dyn, has,
                               *sums)
            self.free, self.static, self.dyn = (o[k].astype(np.float32) for k in ("free", "static", "dyn"))
            return o["born"].astype(np.float32), o["mu"].astype(np.float32), None
        m = O.ds_measgrid(self.G, self.Gz, p.resolution, self.sensor_rel(), p.max_range, p.meas_occ_stddev, pts)
        if sorted_set is None:
            return m["meas_occ"].copy(), None, None
        sums = O.cell_sums(sorted_set["cell"], sorted_set["weight"], sorted_set["vel"], C_)
        o = O.ds_update(p.birth_prob, m["meas_occ"], m["meas_free"], self.occ, self.free, has, *sums)
        self.occ, self.free = o["occ"].astype(np.float32), o["free"].astype(np.float32)
        return o["born"].astype(np.float32), o["mu"].astype(np.float32), o["div"]

    def update_grid(self, t, pts):
        p = self.p
        if self.updated_time > 0:
            dt = float(np.float32(t) - np.float32(self.updated_time))
            self._steady(dt, pts)
        else:
            born, _, _ = self._evidence_and_update(pts, 0.0, None, np.zeros(self.C, np.int32))
            cum = O.exact_scan(born)
            o = O.init_particles(cum, self.P, self.G, p.init_max_velocity, p.particle_min_vel,
                                 O.uniforms(p.seed, self.frame, 2, 0, self.P), prev_cell=self.a["cell"])
            self.a.update(pos=o["pos"], vel=o["vel"], weight=o["weight"], cell=o["cell"])
        self.updated_time = float(t)
        self.frame += 1

    def _steady(self, dt, pts):
        p, P, B = self.p, self.P, self.B
        normals = np.empty(P * 6, np.float32)
        O.oracle().orc_normals_libm(p.seed, self.frame, 0, P, normals)
        pr = O.predict(self.a, normals, self.G, self.Gz, dt, p.persistence_prob, p.stddev_process_noise_position,
                       p.stddev_process_noise_velocity, p.init_max_velocity)
        perm, sk, st, en = O.assign(pr["cell"], self.C)
        srt = {"pos": pr["pos"][perm], "vel": pr["vel"][perm], "weight": pr["weight"][perm], "cell": sk,
               "associated": self.a["associated"][perm]}
        has = (st >= 0).astype(np.int32)
        born, mu, div = self._evidence_and_update(pts, dt, srt, has)
        w = srt["weight"]
        if div is not None:
            d = div[sk].astype(np.float32)
            w = np.where(d > 0, w / np.where(d > 0, d, 1), w).astype(np.float32)
        w = (mu[sk] * w).astype(np.float32)
        cum = O.exact_scan(born)
        b = O.births(born, cum, B, self.G, 0.0, p.init_max_velocity, p.particle_min_vel,
                     O.uniforms(p.seed, self.frame, 3, 0, B), prev_cell=self.birth_cell,
                     prev_assoc=self.birth_assoc)
        self.birth_cell, self.birth_assoc = b["cell"], b["associated"]
        v = srt["vel"]
        m2 = np.float32(p.particle_min_vel) * np.float32(p.particle_min_vel)
        slow = ((v[:, 0] * v[:, 0] + v[:, 1] * v[:, 1]) + v[:, 2] * v[:, 2]) < m2
        w_pen = np.where(slow, np.float32(0), w).astype(np.float32)
        wb = np.where(b["slow"] > 0, np.float32(0), b["weight"]).astype(np.float32)
        anc, _, jmax = O.resample(w_pen, wb, p.seed, self.frame)
        pers = anc < P
        ia, ib = np.minimum(anc, P - 1), np.maximum(anc - P, 0)
        for k, bk in (("pos", "pos"), ("vel", "vel"), ("cell", "cell"), ("associated", "associated")):
            sp, sb = srt[k], b[bk]
            self.a[k] = np.where(pers[:, None] if sp.ndim == 2 else pers, sp[ia], sb[ib])
        self.a["weight"] = np.full(P, np.float32(jmax) / np.float32(P), np.float32)
