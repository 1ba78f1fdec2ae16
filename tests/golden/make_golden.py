"""Generate the golden fixtures in tests/golden/ from the reference itself.

Run where the reference tree is present (by default a folder named
``reference`` beside this repository; override with NOZOMI_REFERENCE_ROOT):

    python tests/golden/make_golden.py [ingestion | faces | collision]

(``ingestion`` regenerates only tests/golden/ingestion.npz, ``faces`` only
tests/golden/dwi_faces.npz, ``collision`` only tests/golden/collision.npz.)  The reference's own Python engine (DiffSim3d / DwiSim3d / SimGeometry3D,
simulation_toolkit/simulation_engine/) is imported with a host stand-in for
pycuda (oracle/fake_pycuda.py); its ``SourceModule`` compiles the reference's
own template-substituted kernel source (sim3d_kernel.cu) for the CPU.  Draws are
injected into the reference's curand calls: a seeded normal table, or the
oracle's counter-based Philox stream (walker, step, draw).  The reference's
own waveform and substrate helpers (waveforms.py, utils/adjust_geometry.py,
DiffSim3d.set_segments) build the inputs.  Every fixture records the inputs,
the draws' description and the reference's outputs.
"""
from __future__ import annotations

import importlib.util
import os
import random
import sys
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(REPO))

from oracle import fake_pycuda  # noqa: E402
from oracle.build import REFERENCE_ROOT  # noqa: E402

OUT = Path(__file__).resolve().parent


def _load_reference():
    fake_pycuda.install()
    sys.path.insert(0, str(REFERENCE_ROOT))
    from simulation_toolkit.simulation_engine import diffsim3d, geometry  # noqa: F401
    spec = importlib.util.spec_from_file_location(
        "ref_waveforms", REFERENCE_ROOT / "simulation_toolkit/simulation_engine/waveforms.py")
    wf = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(wf)
    spec = importlib.util.spec_from_file_location(
        "ref_adjust_geometry", REFERENCE_ROOT / "simulation_toolkit/utils/adjust_geometry.py")
    ag = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(ag)
    return diffsim3d, geometry, wf, ag


class _InRef:
    """cwd = reference root (diffsim3d.py opens its kernel by relative path)."""

    def __enter__(self):
        self.cwd = os.getcwd()
        os.chdir(REFERENCE_ROOT)

    def __exit__(self, *exc):
        os.chdir(self.cwd)


def _geom_arrays(sim):
    return dict(spheres=np.asarray(sim.geom.spheres, np.float64), nstructures=sim.geom.nstructures,
                L=np.array([sim.geom.Lx, sim.geom.Ly, sim.geom.Lz], np.float64),
                nseg=np.array([sim.nsegx, sim.nsegy, sim.nsegz], np.int64),
                dL=np.array([sim.pars["dLx"], sim.pars["dLy"], sim.pars["dLz"]], np.float64),
                K=sim.spheres_per_segment, segments=np.asarray(sim.segments, np.int32),
                D=np.array([s.D for s in sim.geom.structures], np.float32),
                T2=np.array([s.T2 for s in sim.geom.structures], np.float32))


def narrow_case(ds3, geo, name, L, structs, targets, nseg, N, nt, dt, D, seed):
    """randomWalk3d through DiffSim3d.step (the reference's tests' path)."""
    random.seed(seed)
    sg3 = geo.SimGeometry3D(*L, D, 100, 1)
    for (sx, sy, sz, sr) in structs:
        sg3.add_structure(geo.Structure3D(np.asarray(sx), np.asarray(sy), np.asarray(sz), np.asarray(sr), D, 100, 1))
    with _InRef():
        sim = ds3.DiffSim3d(sg3, N)
        sim.set_segments(*nseg)
        fake_pycuda.set_philox(seed, 0, 0)
        sim.setup(structures=targets)
        x0 = sim.spins.astype(np.float32).copy()
        fake_pycuda.reset_step(0)
        for _ in range(nt):
            sim.step(dt)
    np.savez_compressed(OUT / f"{name}.npz", kind="narrow", rng="philox", key=seed,
                        N=N, nt=nt, dt=np.float32(dt), x0=x0, targets=np.asarray(targets),
                        spins=sim.spins_d.get(), spins0=sim.spins0_d.get(), sig=sim.sig_d.get()[0],
                        **_geom_arrays(sim))
    print("wrote", name)


def beaded_axon_c1(ag, rng, n=40, Lz=40.0):
    """One beaded axon: n spheres on the z axis at 1 um spacing, radii U[0.5, 1.5],
    z-periodic images from utils/adjust_geometry.py:create_pad (pad 50)."""
    z = -Lz / 2 + 0.5 + np.arange(n, dtype=np.float64)
    r = rng.uniform(0.5, 1.5, n)
    fib = np.zeros((n, 5))
    fib[:, 2], fib[:, 3] = z, r
    return ag.create_pad(fib.copy(), fib.copy(), Lz)


def dwi_case(ds3, geo, wf, name, L, structs, targets, nseg, N, gwave, dirs, D, key, custom_x0=None,
             three_axis=False):
    """randomWalk3d_phase_multidirr (or randomWalk3d_phase) through
    DwiSim3d.simulate_multi_directions (simulate), Philox-injected draws."""
    random.seed(key)
    sg3 = geo.SimGeometry3D(*L, D, 100, 1)
    for st in structs:
        sx, sy, sz, sr = st[:4]
        Ds = st[4] if len(st) > 4 else D
        sg3.add_structure(geo.Structure3D(np.asarray(sx), np.asarray(sy), np.asarray(sz), np.asarray(sr), Ds, 100, 1))
    with _InRef():
        sim = ds3.DwiSim3d(sg3, N, diffdir=None if three_axis else np.asarray(dirs))
        sim.set_segments(*nseg)
        fake_pycuda.set_philox(key, 0, 0)
        sim.setup(structures=targets)
        if custom_x0 is not None:
            sim.spins = custom_x0.astype(np.float32)
            sim.spins_d = fake_pycuda.GPUArray(sim.spins.copy())
            sim.spins0_d = sim.spins_d.copy()
        x0 = sim.spins_d.get().copy()
        fake_pycuda.reset_step(0)
        log = []
        fake_pycuda.record_scalars(log)
        phase = sim.simulate(gwave) if three_axis else sim.simulate_multi_directions(gwave)
        fake_pycuda.record_scalars(None)
    sc = np.asarray(log, np.float32)  # per launch: dt, G, G_area
    np.savez_compressed(OUT / f"{name}.npz", kind="dwi", rng="philox", key=key, N=N, nt=len(gwave.wave),
                        dt=np.float32(gwave.dt), wave=np.asarray(gwave.wave, np.float64),
                        G=sc[:, 1], Garea=sc[:, 2], dirs=np.asarray(dirs, np.float32),
                        x0=x0, targets=np.asarray([] if targets is None else targets),
                        spins=sim.spins_d.get(), spins0=sim.spins0_d.get(), phase=phase,
                        three_axis=three_axis, **_geom_arrays(sim))
    print("wrote", name)


def segments_cases(ds3, geo):
    rng = np.random.default_rng(11)
    out = {}
    for i, (L, nseg, S) in enumerate([((10, 10, 10), (1, 1, 1), 25), ((10, 10, 10), (2, 2, 3), 40),
                                      ((12, 8, 20), (3, 2, 5), 120), ((7, 7, 7), (4, 4, 4), 60)]):
        sg3 = geo.SimGeometry3D(*L, 2.0, 100, 1)
        for k in range(3):
            m = S // 3
            sx = rng.uniform(-L[0] / 2, L[0] / 2, m)
            sy = rng.uniform(-L[1] / 2, L[1] / 2, m)
            sz = rng.uniform(-L[2] / 2, L[2] / 2, m)
            sr = rng.uniform(0.2, 1.5, m)
            sg3.add_structure(geo.Structure3D(sx, sy, sz, sr, 2.0, 100, 1))
        with _InRef():
            sim = ds3.DiffSim3d(sg3, 1000)
            sim.set_segments(*nseg)
        out[f"case{i}_spheres"] = np.asarray(sg3.spheres, np.float64)
        out[f"case{i}_L"] = np.array(L, np.float64)
        out[f"case{i}_nseg"] = np.array(nseg)
        out[f"case{i}_K"] = sim.spheres_per_segment
        out[f"case{i}_segments"] = np.asarray(sim.segments, np.int32)
    out["ncase"] = 4
    np.savez_compressed(OUT / "segments.npz", **out)
    print("wrote segments")


def waveform_cases(wf):
    out = {}
    pg = wf.PGDiffWaveform(20.0, 10.0, 30.0, time_step=0.01)
    out["pgse_20_10_30_dt01"] = pg.wave
    out["pgse_20_10_30_dt01_b1"] = pg.calculate_bvalue_from_wave()
    pg5 = wf.PGDiffWaveform(20.0, 10.0, 30.0, time_step=0.005)
    out["pgse_20_10_30_dt005"] = pg5.wave
    out["pgse_20_10_30_dt005_b1"] = pg5.calculate_bvalue_from_wave()
    pg2 = wf.PGDiffWaveform(40.0, 10.0, 78.0, time_step=0.002)
    out["pgse_40_10_78_dt002"] = pg2.wave
    og = wf.CosineOGDiffWaveform(2, 50.0, 1.0, 60.0, time_step=0.01)
    out["cos_ogse_2_50_60_dt01"] = og.wave
    out["cos_ogse_2_50_60_dt01_b1"] = og.calculate_bvalue_from_wave()
    ap = wf.ApodizedCosineOGSEWaveform(2, 20.0, te=50.0, time_step=0.01)
    out["apod_ogse_2_20_50_dt01"] = ap.wave
    out["apod_ogse_2_20_50_dt01_b1"] = ap.calculate_bvalue_from_wave()
    np.savez_compressed(OUT / "waveforms.npz", **out)
    print("wrote waveforms")


def seeding_case(geo):
    """seedSpinsKernel's accept rule for injected uniforms (one launch)."""
    import ctypes
    rng = np.random.default_rng(21)
    L = (6.0, 5.0, 7.0)
    structs = []
    for k in range(3):
        m = 6
        structs.append((rng.uniform(-2.5, 2.5, m), rng.uniform(-2, 2, m), rng.uniform(-3, 3, m), rng.uniform(0.5, 1.5, m)))
    sg3 = geo.SimGeometry3D(*L, 2.0, 100, 1)
    for s in structs:
        sg3.add_structure(geo.Structure3D(*s, 2.0, 100, 1))
    N = 4000
    u = rng.uniform(0, 1, (N, 3)).astype(np.float32)
    u[:8] = [[0, 0.5, 0.5], [1, 0.5, 0.5], [0.5, 0, 0.5], [0.5, 1, 0.5], [0.5, 0.5, 0], [0.5, 0.5, 1],
             [0.5, 0.5, 0.5], [0.25, 0.75, 0.5]]
    code_pars = {"nspins": N, "nspheres": sg3.nsphere, "nspheres_per_seg": sg3.nsphere, "nstructures": 3,
                 "Lx": 6.0, "Ly": 5.0, "Lz": 7.0, "dLx": 6.0, "dLy": 5.0, "dLz": 7.0, "nLx": 1, "nLy": 1, "nLz": 1,
                 "D": "2,2,2,2", "T2": "100,100,100,100", "ndiffdir": 3}
    from oracle.build import build_reference_kernel, substitute_reference
    lib = ctypes.CDLL(str(build_reference_kernel(substitute_reference(code_pars))))
    all_sph = np.vstack([np.vstack([s[0], s[1], s[2], s[3]]).T for s in structs]).astype(np.float32).ravel()
    counts = np.array([6, 6, 6, 0], np.int32)
    out = {"spheres": np.asarray(sg3.spheres, np.float64), "L": np.array(L), "u": u}
    lib.ref_set_uniforms.argtypes = [ctypes.c_void_p, ctypes.c_int]
    lib.ref_set_uniforms(u.ctypes.data, 3)
    for tname, tg in [("intra", [0, 1, 2]), ("extra", [3]), ("s1", [1]), ("all", [0, 1, 2, 3])]:
        idx = np.array(tg, np.int32)
        pos = np.zeros(3 * N, np.float32)
        status = np.ones(N, np.int32)
        lib.ref_run_seed(ctypes.c_int(1), ctypes.c_int(N), ctypes.c_int(N), ctypes.c_int(4),
                         ctypes.c_void_p(all_sph.ctypes.data), ctypes.c_void_p(counts.ctypes.data),
                         ctypes.c_void_p(pos.ctypes.data), ctypes.c_int(len(idx)), ctypes.c_void_p(idx.ctypes.data),
                         ctypes.c_float(L[0]), ctypes.c_float(L[1]), ctypes.c_float(L[2]), ctypes.c_uint(7),
                         ctypes.c_void_p(status.ctypes.data))
        out[f"{tname}_targets"] = idx
        out[f"{tname}_accept"] = status == 0
        out[f"{tname}_pos"] = pos.reshape(3, N)
    lib.ref_set_uniforms(None, 0)
    np.savez_compressed(OUT / "seeding.npz", **out)
    print("wrote seeding")


def ingestion_case(ag, tmpdir):
    """The simulation driver's substrate ingestion (simulation_main.py:37-49):
    the pickle read by common_utils.import_array_geometry_full_path, split at
    z == L/2 by split_matrix_to_list, z-padded by createBoundaryZ.  Fibres run
    from z = -L/2 to L/2; some continue through the z face as another fibre
    (a tilted chain A -> B -> C -> A), some as themselves, one has no partner."""
    import pickle
    import torch
    import simulation_toolkit.toolkit_params as params
    import simulation_toolkit.utils.common_utils as cu
    rng = np.random.default_rng(31)
    L = 20.0
    fibres = []
    pts = [(-6.0, -4.0), (-3.0, 1.0), (2.0, 5.0)]  # the chain's entry points
    for i, (a, b) in enumerate(zip(pts, pts[1:] + pts[:1])):  # A -> B -> C -> A
        fibres.append((a, b))
    fibres.append(((5.0, -5.0), (5.0, -5.0)))  # its own partner
    fibres.append(((8.0, 8.0), (7.5, 8.5)))    # no fibre starts at (7.5, 8.5)
    rows = []
    for fid, ((x0, y0), (x1, y1)) in enumerate(fibres):
        n = int(rng.integers(45, 70))
        t = np.linspace(0.0, 1.0, n)
        z = -L / 2 + t * L
        z[-1] = L / 2  # the split marker: exactly L/2
        x, y = x0 + t * (x1 - x0), y0 + t * (y1 - y0)
        x[-1], y[-1] = x1, y1
        r = rng.uniform(0.4, 1.2, n)
        rows.append(np.stack([x, y, z, r, np.full(n, float(fid))], axis=1))
    A = np.concatenate(rows)
    path = Path(tmpdir) / "substrate.pkl"
    with open(path, "wb") as f:
        pickle.dump([torch.from_numpy(A), L], f, protocol=pickle.HIGHEST_PROTOCOL)
    arr, Lr = cu.import_array_geometry_full_path(str(path))
    params.BOX_LENGTH = Lr
    fl = cu.split_matrix_to_list(arr)
    out = ag.createBoundaryZ(fl, Lr)
    np.savez_compressed(OUT / "ingestion.npz", matrix=A, L=L, lengths=np.array([len(f) for f in out]),
                        fibres=np.concatenate(out))


def faces_case(ds3, geo, wf):
    """Walkers started on the box and cell boundaries: a non-cubic 6 x 5 x 7 um
    box with 4 x 3 x 5 cells (edges 1.5, 5/3 and 1.4 um, none a power of two),
    spheres of two structures crossing every face, 10 directions.  Of 1000
    walkers, 400 start on a face, an edge or a corner of the box, exactly or
    one float32 ulp inside or outside, and 200 exactly on interior cell
    boundaries (x = -L/2 + k dL in float32); the rest uniformly in the box."""
    rng = np.random.default_rng(11)
    L = np.array([6.0, 5.0, 7.0])
    structs = []
    for k, Dk in enumerate((1.2, 0.8)):
        m = 10
        c = rng.uniform(-0.5, 0.5, (3, m)) * L[:, None]
        for i in range(6):  # one sphere centred on each face
            c[i // 2, i] = (1 if i % 2 else -1) * L[i // 2] / 2
        structs.append((c[0], c[1], c[2], rng.uniform(0.5, 1.3, m), Dk))
    N = 1000
    x0 = (rng.uniform(-0.5, 0.5, (3, N)) * L[:, None]).astype(np.float32)
    half = (L / 2).astype(np.float32)
    for w in range(400):
        nax = 1 + w % 3  # a face, an edge or a corner
        axes = rng.choice(3, nax, replace=False)
        for a in axes:
            v = half[a] if rng.random() < 0.5 else -half[a]
            step = (w // 3) % 3  # exactly, one ulp toward +inf, one toward -inf
            if step == 1:
                v = np.nextafter(v, np.float32(np.inf))
            elif step == 2:
                v = np.nextafter(v, np.float32(-np.inf))
            x0[a, w] = v
    nseg = (4, 3, 5)
    dL = (L / np.array(nseg)).astype(np.float32)
    for w in range(400, 600):
        a = w % 3
        k = rng.integers(1, nseg[a])
        x0[a, w] = np.float32(-half[a] + np.float32(k) * dL[a])
    dirs = rng.standard_normal((3, 10))
    dirs /= np.linalg.norm(dirs, axis=0)
    pg = wf.PGDiffWaveform(2.0, 1.0, 3.0, time_step=0.01)
    dwi_case(ds3, geo, wf, "dwi_faces", tuple(L), structs, None, nseg, N, pg, dirs, 2.0, 505, custom_x0=x0)


def collision_case():
    """collision.npz: the reference's own collide_spheres_gpu
    (substrate_generator/helper/CollisionDetection.py, loaded by file path,
    run on CPU tensors) on a seeded 500-axon bundle whose sphere centres are
    jittered (so that axons overlap), spheres inside the box only, for buff
    0 and 0.05 um, with the closest call's distance from the threshold."""
    import torch
    from nozomi_b200.substrates import axon_bundle
    from oracle.collide_oracle import margin
    spec = importlib.util.spec_from_file_location(
        "ref_collision", REFERENCE_ROOT / "simulation_toolkit/substrate_generator/helper/CollisionDetection.py")
    cd = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(cd)
    sub = axon_bundle(500, seed=11)
    rng = np.random.default_rng(12)
    rows = []
    for k, f in enumerate(sub.fibers):
        f = np.asarray(f, np.float64)
        inside = np.all(np.abs(f[:, :3]) <= np.array(sub.L) / 2, axis=1)
        f = f[inside]
        rows.append(np.column_stack([f[:, :4], np.full(len(f), float(k))]))
    A = np.concatenate(rows)
    A[:, :2] += rng.normal(0.0, 0.3, (len(A), 2))
    A[:, :2] = np.clip(A[:, :2], -np.array(sub.L[:2]) / 2, np.array(sub.L[:2]) / 2)
    pos = torch.from_numpy(A[:, :3].astype(np.float32))
    r = torch.from_numpy(A[:, 3].astype(np.float32))
    fid = torch.from_numpy(A[:, 4].astype(np.float32))
    Lx, Ly, Lz = (torch.tensor(float(v), dtype=torch.float32) for v in sub.L)
    out = {"pos": pos.numpy(), "radii": r.numpy(), "fiber_id": fid.numpy(), "L": np.array(sub.L, np.float32)}
    for i, buff in enumerate((0.0, 0.05)):
        pairs = cd.collide_spheres_gpu(pos, r, fid, Lx, Ly, Lz, torch.tensor([buff], dtype=torch.float32))
        out[f"buff{i}"] = np.float32(buff)
        out[f"pairs{i}"] = pairs.numpy().astype(np.int32)
        out[f"margin{i}"] = margin(pos.numpy(), r.numpy(), fid.numpy(), buff)
        print("collision", buff, pairs.shape[0], "pairs, closest call", out[f"margin{i}"])
    np.savez_compressed(OUT / "collision.npz", **out)


def main():
    if sys.argv[1:] == ["collision"]:
        collision_case()
        return
    ds3, geo, wf, ag = _load_reference()
    if sys.argv[1:] == ["ingestion"]:
        import tempfile
        with tempfile.TemporaryDirectory() as d:
            ingestion_case(ag, d)
        return
    if sys.argv[1:] == ["faces"]:
        faces_case(ds3, geo, wf)
        return
    import tempfile
    with tempfile.TemporaryDirectory() as d:
        ingestion_case(ag, d)
    segments_cases(ds3, geo)
    waveform_cases(wf)
    seeding_case(geo)

    one = ([0.0], [0.0], [0.0], [1.0])
    nsph = 20
    sz = np.arange(-nsph / 2 - 2, nsph / 2 + 3) * 10 / nsph
    sy = np.sin(2 * np.pi * np.arange(-2, nsph + 3) / nsph) * 0.25
    chain = (np.zeros_like(sz), sy, sz, np.ones_like(sz))
    narrow_case(ds3, geo, "narrow_sphere_in", (10, 10, 10), [one], [0], (1, 1, 1), 1000, 300, 0.002, 3.0, 1)
    narrow_case(ds3, geo, "narrow_sphere_out", (10, 10, 10), [one], [1], (2, 2, 2), 1000, 300, 0.002, 3.0, 2)
    narrow_case(ds3, geo, "narrow_chain_in", (10, 10, 10), [chain], [0], (1, 1, 1), 1000, 300, 0.002, 3.0, 3)
    narrow_case(ds3, geo, "narrow_chain_out", (10, 10, 10), [chain], [1], (2, 2, 3), 1000, 300, 0.002, 3.0, 4)
    # two wavy chains across the x faces with z-periodic images (test_03 geometry)
    z = np.linspace(-5, 5, num=200)
    z = np.concatenate((z[-30:-1] - 10, z, z[1:30] + 10))
    y = np.sin(2 * np.pi * z / 10)
    px = (np.concatenate((np.full(z.shape, 5.0), np.full(z.shape, -5.0))), np.concatenate((y, y)),
          np.concatenate((z, z)), np.ones(2 * z.size))
    narrow_case(ds3, geo, "narrow_periodic_in", (10, 10, 10), [px], [0], (3, 3, 3), 1000, 300, 0.002, 3.0, 5)

    # C1 substrate and protocol: one beaded axon, PGSE 20/10/30 at dt = 10 us, x and z
    rng = np.random.default_rng(1)
    ax = beaded_axon_c1(ag, rng)
    c1 = (ax[:, 0], ax[:, 1], ax[:, 2], ax[:, 3])
    pg = wf.PGDiffWaveform(20.0, 10.0, 30.0, time_step=0.01)
    dirs_xz = np.array([[1.0, 0.0], [0.0, 0.0], [0.0, 1.0]])
    dwi_case(ds3, geo, wf, "dwi_c1", (8.0, 8.0, 40.0), [c1], [0], (1, 1, 1), 1000, pg, dirs_xz, 2.0, 101)
    dwi_case(ds3, geo, wf, "dwi_c1_cells", (8.0, 8.0, 40.0), [c1], [0], (2, 2, 8), 1000, pg, dirs_xz, 2.0, 102)

    # overlapping structures, mixed seeding, 10 directions, short PGSE, walkers
    # placed on surfaces and in the tolerance shells
    rng = np.random.default_rng(7)
    structs = []
    for k in range(3):
        m = 8
        structs.append((rng.uniform(-2.5, 2.5, m), rng.uniform(-2.5, 2.5, m), rng.uniform(-2.5, 2.5, m),
                        rng.uniform(0.4, 1.4, m), [1.0, 1.5, 0.7][k]))
    dirs = rng.standard_normal((3, 10))
    dirs /= np.linalg.norm(dirs, axis=0)
    pg_short = wf.PGDiffWaveform(2.0, 1.0, 3.0, time_step=0.01)
    N = 1000
    x0 = rng.uniform(-3, 3, (3, N))
    allsph = np.concatenate([np.vstack(s[:4]) for s in structs], axis=1)
    for w in range(300):
        s = w % allsph.shape[1]
        v = rng.standard_normal(3)
        v /= np.linalg.norm(v)
        off = [0.0, 1e-4, -1e-4, 5e-5, -5e-5, 2e-4][w % 6]
        x0[:, w] = allsph[:3, s] + (allsph[3, s] + off) * v
    x0 = np.clip(x0, -2.999, 2.999)
    dwi_case(ds3, geo, wf, "dwi_overlap", (6.0, 6.0, 6.0), structs, None, (2, 3, 2), N, pg_short, dirs, 2.5, 303,
             custom_x0=x0)
    dwi_case(ds3, geo, wf, "dwi_overlap_3axis", (6.0, 6.0, 6.0), structs, None, (1, 1, 1), N, pg_short,
             np.eye(3), 2.5, 304, custom_x0=x0, three_axis=True)
    faces_case(ds3, geo, wf)


if __name__ == "__main__":
    main()
