"""Seeded synthetic LiDAR scenes that stand in for the reference's rosbags (data/*.bag are
not in the reference checkout).

A scene is a ground plane, static and moving axis-aligned cuboids, and an enclosing
cylindrical wall at the sensor's maximum range (so every beam returns, as a bag replayed into
the node would deliver a fixed-size cloud). A multi-beam LiDAR with uniform azimuth steps
and evenly spread elevations casts rays from the sensor; ranges get Gaussian noise. Points
are returned sensor-centred and map-axis aligned, the frame DOM::updateGrid expects
(k3dom_node.cpp:73-85).

The named configurations mirror the benchmark configurations of this project:
  config0: 64x64x16 @ 0.2 m, P=262144, B=65536, one 32-beam scan of 30000 returns.
  config1: 256x256x32 @ 0.1 m, P=4194304, B=1048576, 64-beam scans of 120000 returns,
           ego motion 0-2 m/s, 20 static + 20 moving cuboids at 0-3 m/s, 10 Hz.
  config2: config1's shape with the DS-PHD/MIB variant.
  config3: 16 independent scenes for the batched update, per-scene seeds: grids G x G x Gz at
           0.1 m with G uniform in 64..256 and Gz in 16..32, P = 2^u with u uniform in [18, 22],
           B = P / 4, 10,000-200,000 points per scan; contents as config1 (20 static + 20 moving
           cuboids, ego motion 0-2 m/s) scaled to each grid.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np


@dataclasses.dataclass
class Box:
    center: np.ndarray  # (3,) at t = 0, world frame [m]
    half: np.ndarray    # (3,)
    vel: np.ndarray     # (3,) [m/s]


class Scene:
    def __init__(self, seed: int = 0, n_static: int = 2, n_moving: int = 0, side=(1.0, 2.0), speed=(0.5, 1.5),
                 ego_speed=(0.0, 0.0), extent: float = 6.0, ground_z: float = -1.5, max_range: float = 12.8,
                 beams: int = 32, elev_deg=(-25.0, 15.0), range_noise: float = 0.02):
        rng = np.random.Generator(np.random.PCG64(seed))
        self.seed = seed
        self.ground_z = ground_z
        self.max_range = max_range
        self.beams = beams
        self.elev = np.deg2rad(np.linspace(elev_deg[0], elev_deg[1], beams))
        self.range_noise = range_noise
        self.boxes: list[Box] = []
        for k in range(n_static + n_moving):
            moving = k >= n_static
            h = rng.uniform(side[0], side[1], size=3) / 2.0
            # keep boxes out of a 1.5 m radius around the start position
            while True:
                c = rng.uniform(-extent, extent, size=2)
                if np.hypot(*c) > 1.5 + h[:2].max():
                    break
            center = np.array([c[0], c[1], ground_z + h[2]])
            v = np.zeros(3)
            if moving:
                sp = rng.uniform(speed[0], speed[1])
                hd = rng.uniform(0.0, 2.0 * math.pi)
                v = np.array([sp * math.cos(hd), sp * math.sin(hd), 0.0])
            self.boxes.append(Box(center, h, v))
        sp = rng.uniform(ego_speed[0], ego_speed[1])
        hd = rng.uniform(0.0, 2.0 * math.pi)
        self.ego_vel = np.array([sp * math.cos(hd), sp * math.sin(hd), 0.0])
        self._noise_seed = int(rng.integers(0, 2**63 - 1))

    def sensor_pos(self, t: float) -> np.ndarray:
        return self.ego_vel * t

    def scan(self, frame: int, t: float, n_points: int, sensor_offset=None,
             az_offset: float = 0.0) -> tuple[np.ndarray, np.ndarray]:
        """(sensor position in the world [m], points (n, 3) float32 relative to the sensor).
        sensor_offset moves the sensor off its trajectory; az_offset rotates the beam pattern."""
        s = self.sensor_pos(t)
        if sensor_offset is not None:
            s = s + np.asarray(sensor_offset, np.float64)
        n_az = -(-n_points // self.beams)
        az = np.linspace(0.0, 2.0 * math.pi, n_az, endpoint=False) + az_offset
        el = self.elev
        ce, se = np.cos(el), np.sin(el)
        d = np.stack([np.outer(ce, np.cos(az)), np.outer(ce, np.sin(az)), np.outer(se, np.ones_like(az))],
                     axis=-1).reshape(-1, 3)[:n_points]
        # enclosing wall at max_range (horizontal distance)
        horiz = np.hypot(d[:, 0], d[:, 1])
        t_hit = np.where(horiz > 1e-9, self.max_range / np.maximum(horiz, 1e-9), np.inf)
        # ground
        with np.errstate(divide="ignore", invalid="ignore"):
            tg = np.where(d[:, 2] < 0, (self.ground_z - s[2]) / d[:, 2], np.inf)
        t_hit = np.minimum(t_hit, np.where(tg > 0, tg, np.inf))
        # cuboids (slab test); fmin/fmax ignore the NaN of 0 * inf on axis-parallel rays
        d32 = d.astype(np.float32)
        with np.errstate(divide="ignore", invalid="ignore"):
            inv = (1.0 / d32).astype(np.float32)
        for b in self.boxes:
            c = (b.center + b.vel * t - s).astype(np.float32)
            h = b.half.astype(np.float32)
            with np.errstate(invalid="ignore"):
                t0 = (c - h) * inv
                t1 = (c + h) * inv
            lo = np.fmin(t0, t1)
            hi = np.fmax(t0, t1)
            tmin = np.fmax(np.fmax(lo[:, 0], lo[:, 1]), lo[:, 2])
            tmax = np.fmin(np.fmin(hi[:, 0], hi[:, 1]), hi[:, 2])
            ok = (tmax >= tmin) & (tmin > 0) & (tmin < t_hit)
            t_hit = np.where(ok, tmin, t_hit)
        t_hit = np.minimum(t_hit, self.max_range / np.maximum(np.abs(d[:, 2]), 1e-9))
        rng = np.random.Generator(np.random.PCG64([self._noise_seed, frame]))
        r = t_hit + rng.normal(0.0, self.range_noise, size=t_hit.shape)
        pts = (d * r[:, None]).astype(np.float32)
        return s.astype(np.float32), pts


@dataclasses.dataclass
class Config:
    name: str
    variant: str
    params: dict
    scene: Scene
    n_points: int
    frames: int
    dt: float


def _k3dom_params(size, size_z, res, P, B, ls=0.3, sigma=0.1, variant="k3dom", seed=0, max_points=0):
    """Parameter values of config/k3dom.yaml (or dsphdmib.yaml) in index units, as the node
    converts them (k3dom_node.cpp:344-368)."""
    p = dict(size=size, size_z=size_z, resolution=res, particle_count=P, new_born_particle_count=B,
             mass_scale=2.5, persistence_prob=0.99, stddev_process_noise_position=0.01 / res,
             stddev_process_noise_velocity=0.1 / res, birth_prob=0.02, stddev_velocity=4.0 / res,
             init_max_velocity=5.0 / res, particle_min_vel=0.1 / res, sensor_off_x=0.0, sensor_off_y=0.0,
             sensor_off_z=0.0, map_shift_thresh=int(np.float32(1.0) / np.float32(res)), prior_free=0.001,
             prior_static=0.001, prior_dynamic=0.001, prior_occ=0.0, sigma=sigma, ls=ls, gamma=0.99,
             max_range=50.0, meas_occ_stddev=0.1, seed=seed, max_points=max_points)
    if variant == "dsphdmib":
        p.update(particle_min_vel=0.0, prior_free=0.0, prior_static=0.0, prior_dynamic=0.0, prior_occ=0.0)
    return p


def config0(seed: int = 0) -> Config:
    scene = Scene(seed=seed, n_static=0, n_moving=2, side=(1.0, 2.0), speed=(0.5, 1.5), extent=5.0,
                  ground_z=-1.5, max_range=12.8, beams=32, range_noise=0.02)
    return Config("config0", "k3dom", _k3dom_params(12.8, 3.2, 0.2, 262144, 65536, max_points=30000),
                  scene, 30000, 2, 0.1)


def config1(seed: int = 0, variant: str = "k3dom") -> Config:
    scene = Scene(seed=seed, n_static=20, n_moving=20, side=(1.0, 2.0), speed=(0.0, 3.0), ego_speed=(0.0, 2.0),
                  extent=11.0, ground_z=-1.5, max_range=25.6, beams=64, range_noise=0.02)
    return Config("config1" if variant == "k3dom" else "config2", variant,
                  _k3dom_params(25.6, 3.2, 0.1, 4194304, 1048576, variant=variant, max_points=120000),
                  scene, 120000, 100, 0.1)


def config2(seed: int = 0) -> Config:
    return config1(seed, "dsphdmib")


def config3(seed: int = 0, n_scenes: int = 16, variant: str = "k3dom") -> list:
    rng = np.random.Generator(np.random.PCG64([seed, 3]))
    out = []
    for k in range(n_scenes):
        G = int(rng.integers(64, 257))
        Gz = int(rng.integers(16, 33))
        P = int(round(2.0 ** rng.uniform(18.0, 22.0)))
        B = max(1, P // 4)
        n = int(rng.integers(10000, 200001))
        res = 0.1
        size, size_z = G * res, Gz * res
        sc = Scene(seed=seed * 1000 + k, n_static=20, n_moving=20, side=(1.0, 2.0), speed=(0.0, 3.0),
                   ego_speed=(0.0, 2.0), extent=max(2.0, size / 2 - 1.5), ground_z=-1.5, max_range=size,
                   beams=64, range_noise=0.02)
        params = _k3dom_params(size, size_z, res, P, B, variant=variant, seed=5000 + k, max_points=n)
        out.append(Config(f"config3[{k}]", variant, params, sc, n, 100, 0.1))
    return out


@dataclasses.dataclass
class CalibConfig:
    """The differentiable update's calibration problem: training frames (t, sensor, points) and
    held-out scans (sensor, points), all sensor positions in the world frame."""
    name: str
    params: dict
    train: list
    heldout: list
    theta0: tuple


def config4(seed: int = 0, scale: str = "config0", n_heldout: int = 10) -> CalibConfig:
    """config0's grid and scans (initialisation + one update) and 10 held-out 30,000-point scans
    of the scene at the last training time from sensors displaced by up to 0.5 m, with rotated
    beam patterns; theta0 = (ls 0.3 m, sigma 1.0, gamma 0.1, occupied prior 0.01, free prior 0.01).
    scale="config1" uses config1's grid, particle counts and 120,000-point scans instead."""
    base = config0(seed) if scale == "config0" else config1(seed)
    rng = np.random.Generator(np.random.PCG64([seed, 4]))
    params = dict(base.params)
    theta0 = (0.3, 1.0, 0.1, 0.01, 0.01)
    params.update(ls=theta0[0], sigma=theta0[1], gamma=theta0[2], prior_static=theta0[3] / 2,
                  prior_dynamic=theta0[3] / 2, prior_free=theta0[4])
    train = []
    for f in range(2):
        t = 0.1 + f * base.dt
        s, pts = base.scene.scan(f, t, base.n_points)
        train.append((t, s, pts))
    t_last = train[-1][0]
    heldout = []
    for k in range(n_heldout):
        off = rng.uniform(-0.5, 0.5, 3) * np.array([1.0, 1.0, 0.2])
        s, pts = base.scene.scan(100 + k, t_last, 30000 if scale == "config0" else base.n_points,
                                 sensor_offset=off, az_offset=float(rng.uniform(0, 2 * math.pi)))
        heldout.append((s, pts))
    return CalibConfig(f"config4[{scale}]", params, train, heldout, theta0)


def small(seed: int = 0, variant: str = "k3dom", G: int = 32, Gz: int = 8, res: float = 0.2, P: int = 16384,
          B: int = 4096, n_points: int = 2000, n_moving: int = 2, ego: float = 0.0) -> Config:
    """A small scene for parity tests (the CPU oracle finishes in well under a second)."""
    size, size_z = G * res, Gz * res
    scene = Scene(seed=seed, n_static=1, n_moving=n_moving, side=(0.6, 1.2), speed=(0.5, 1.5),
                  ego_speed=(ego, ego), extent=size / 2 - 0.5, ground_z=-0.6, max_range=size / 2 + 1.0,
                  beams=16, elev_deg=(-30.0, 10.0), range_noise=0.02)
    p = _k3dom_params(size, size_z, res, P, B, variant=variant, max_points=n_points)
    return Config(f"small{G}", variant, p, scene, n_points, 4, 0.1)
