"""Generate the golden fixtures tests/golden/{k3dom,dsphdmib}_small.npz and
tests/golden/k3dom_shift_small.npz.

Runs the reference's own CUDA update (oracle/_ref/libref_*.so, built from the reference's
sources by oracle/build_ref.sh) stage by stage on a small seeded synthetic scene, with the
Philox draws injected through the curand shim, and records every stage's inputs and outputs.
Requires a GPU; run from the repository root:

    python tests/golden/make_golden.py [outdir] [--only shift]

The fixtures are committed; the CPU tests (tests/test_oracle_golden.py) check the oracle
against them.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from k3dom_b200 import make_params, scene  # noqa: E402
from k3dom_b200.dom import debug_draws  # noqa: E402
from oracle.binding import Reference  # noqa: E402

SEED = 7
SIZES = dict(G=32, Gz=8, res=0.2, P=8192, B=2048, n_points=1500)
FRAMES = 3


def record_particles(rec, key, d):
    for k, v in d.items():
        rec[f"{key}_{k}"] = v


def run(variant: str, out: Path) -> None:
    cfg = scene.small(seed=SEED, variant=variant, **SIZES)
    cfg.params["seed"] = 1234
    p = make_params(variant, **cfg.params)
    ref = Reference(p, variant)
    rec = {"seed": np.int64(p.seed), "G": np.int32(ref.G), "Gz": np.int32(ref.Gz), "P": np.int32(ref.P),
           "B": np.int32(ref.B), "params": np.frombuffer(bytes(p), np.uint8)}
    t_prev = None
    for f in range(FRAMES):
        t = 0.1 + f * cfg.dt
        s, pts = cfg.scene.scan(f, t, cfg.n_points)
        ref.update_pose(*s)
        rec[f"f{f}_pose"] = s
        rec[f"f{f}_pts"] = pts
        rec[f"f{f}_sensor_rel"] = ref.sensor_rel()
        rec[f"f{f}_t"] = np.float32(t)
        if f == 0:
            rec["f0_cells_in"] = ref.cells()
            rec["f0_prev_cell"] = ref.particles(0)["cell"]
            ref.init_particles(f, pts)
            rec["f0_cells_out"] = ref.cells()
            born = ref.born()
            rec["f0_born"] = born
            rec["f0_born_cum"] = ref.thrust_scan(born)
            if variant == "dsphdmib":
                rec["f0_meas_occ"], rec["f0_meas_free"] = ref.meas()
            record_particles(rec, "f0_init", ref.particles(0))
            rec["f0_init_uniforms"] = debug_draws(p.seed, f, 2, 0, ref.P)
            ref.finish(t, False)
        else:
            dt = np.float32(t) - np.float32(t_prev)
            rec[f"f{f}_dt"] = np.float32(dt)
            # prediction
            record_particles(rec, f"f{f}_pred_in", ref.particles(0))
            rec[f"f{f}_normals"] = debug_draws(p.seed, f, 1, 0, ref.P)
            ref.predict(f, dt)
            record_particles(rec, f"f{f}_pred_out", ref.particles(0))
            # assignment
            ref.assign()
            record_particles(rec, f"f{f}_sorted", ref.particles(0))
            # occupancy update
            rec[f"f{f}_cells_in"] = ref.cells()
            ref.occupancy(dt, pts)
            rec[f"f{f}_cells_occ"] = ref.cells()
            born = ref.born()
            rec[f"f{f}_born"] = born
            if variant == "dsphdmib":
                rec[f"f{f}_meas_occ"], rec[f"f{f}_meas_free"] = ref.meas()
                rec[f"f{f}_sorted_after_occ_weight"] = ref.particles(0)["weight"]
            # persistent particles
            ref.persistent()
            rec[f"f{f}_reweighted"] = ref.particles(0)["weight"]
            rec[f"f{f}_cells_pers"] = ref.cells()
            # births
            prev_birth = ref.particles(2)
            rec[f"f{f}_birth_prev_cell"] = prev_birth["cell"]
            rec[f"f{f}_birth_prev_assoc"] = prev_birth["associated"]
            rec[f"f{f}_born_cum"] = ref.thrust_scan(born)
            rec[f"f{f}_birth_uniforms"] = debug_draws(p.seed, f, 3, 0, ref.B)
            ref.births(f)
            record_particles(rec, f"f{f}_birth", ref.particles(2))
            # moments; the reference's own FP32 prefix sums behind statisticalMomentsKernel2
            # and updatePersistentParticlesKernel2 (subtract() of include/common/common.h:20-28)
            srt = ref.particles(0)
            wv = (srt["weight"][:, None] * srt["vel"]).astype(np.float32)
            rec[f"f{f}_wv_cum"] = np.stack([ref.thrust_scan(wv[:, k]) for k in range(3)], 1)
            rec[f"f{f}_postw_cum"] = ref.thrust_scan(rec[f"f{f}_sorted_weight"] if variant == "k3dom"
                                                     else rec[f"f{f}_sorted_after_occ_weight"])
            ref.moments()
            rec[f"f{f}_cells_mom"] = ref.cells()
            # resampling
            ref.resampling(f)
            sorted_after = ref.particles(0)
            births_after = ref.particles(2)
            rec[f"f{f}_joint_sorted_w"] = sorted_after["weight"]
            rec[f"f{f}_joint_birth_w"] = births_after["weight"]
            joint = np.concatenate([sorted_after["weight"], births_after["weight"]])
            rec[f"f{f}_joint_cum"] = ref.thrust_scan(joint)
            record_particles(rec, f"f{f}_next", ref.particles(1))
            ref.finish(t, True)
        t_prev = t
    ref.close()
    np.savez_compressed(out, **rec)
    print(f"wrote {out} ({out.stat().st_size / 1e6:.2f} MB)")


SHIFT_FRAMES = 7
SHIFT_EGO = 6.0  # m/s: 0.6 m = 3 voxels per frame at 0.2 m, so the 5-voxel threshold fires every 2nd frame


def run_shift(out: Path) -> None:
    """Ego motion: the sensor moves 0.6 m per frame, so DOM_c::updatePose shifts the map
    (src/common/dom.cu:111-158; moveMapKernel / moveParticlesKernel,
    src/common/kernel/ego_motion_compensation.cu:12-41) every other frame. Recorded around each
    updatePose: the map centre, the 68-byte cells and the particle positions before and after;
    and the prediction that follows (its input is the shifted set)."""
    variant = "k3dom"
    cfg = scene.small(seed=SEED + 4, variant=variant, ego=SHIFT_EGO, **SIZES)
    cfg.params["seed"] = 4321
    p = make_params(variant, **cfg.params)
    ref = Reference(p, variant)
    rec = {"seed": np.int64(p.seed), "G": np.int32(ref.G), "Gz": np.int32(ref.Gz), "P": np.int32(ref.P),
           "B": np.int32(ref.B), "params": np.frombuffer(bytes(p), np.uint8)}
    t_prev = None
    for f in range(SHIFT_FRAMES):
        t = 0.1 + f * cfg.dt
        s, pts = cfg.scene.scan(f, t, cfg.n_points)
        rec[f"f{f}_pose"] = np.asarray(s, np.float32)
        rec[f"f{f}_center_before"] = ref.center()
        if f > 0:
            rec[f"f{f}_cells_before"] = ref.cells()
            rec[f"f{f}_pos_before"] = ref.particles(0)["pos"]
        ref.update_pose(*s)
        rec[f"f{f}_center_after"] = ref.center()
        if f == 0:
            ref.init_particles(f, pts)
            ref.finish(t, False)
        else:
            rec[f"f{f}_cells_after"] = ref.cells()
            a = ref.particles(0)
            rec[f"f{f}_pos_after"] = a["pos"]
            for k in ("vel", "weight"):
                rec[f"f{f}_pred_in_{k}"] = a[k]
            idx = np.arange(ref.C, dtype=np.int32)
            rec[f"f{f}_coord_idx"] = idx
            rec[f"f{f}_coords"] = ref.index_to_coord(idx)
            dt = np.float32(t) - np.float32(t_prev)
            rec[f"f{f}_dt"] = np.float32(dt)
            rec[f"f{f}_normals"] = debug_draws(p.seed, f, 1, 0, ref.P)
            ref.predict(f, dt)
            out_p = ref.particles(0)
            for k in ("pos", "vel", "weight", "cell"):
                rec[f"f{f}_pred_out_{k}"] = out_p[k]
            ref.assign()
            ref.occupancy(dt, pts)
            ref.persistent()
            ref.births(f)
            ref.moments()
            ref.resampling(f)
            ref.finish(t, True)
        t_prev = t
    ref.close()
    np.savez_compressed(out, **rec)
    print(f"wrote {out} ({out.stat().st_size / 1e6:.2f} MB)")


def main(argv):
    args = [a for a in argv[1:] if not a.startswith("--")]
    only = argv[argv.index("--only") + 1] if "--only" in argv else None
    if only:
        args = [a for a in args if a != only]
    outdir = Path(args[0]) if args else Path(__file__).resolve().parent
    outdir.mkdir(parents=True, exist_ok=True)
    if only in (None, "small"):
        for v in ("k3dom", "dsphdmib"):
            run(v, outdir / f"{v}_small.npz")
    if only in (None, "shift"):
        run_shift(outdir / "k3dom_shift_small.npz")
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv))
