"""GPU parity: the CUDA kernels against the oracle and the reference's own
outputs (golden fixtures), through the C ABI.

Bar: bit-exact for cell lists, labels, collision counts, positions, spins0,
phase and Phi (same draws, same cell lists); T2 signal within 2e-6 relative
(expf ulps); FP64 signal sums within 1e-9 absolute of the oracle's (FP32 sincos
per walker, different summation order).
"""
import numpy as np
import pytest

from tests._fixtures import DWI, EDGE, NARROW, dirs_of, load, oracle_geometry
from oracle import oracle as oz
from oracle.cells_oracle import cells_members, segments_reference

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eng():
    from nozomi_b200 import engine
    engine.require_cuda()
    return engine


def _dev(a, dtype=None):
    t = torch.from_numpy(np.ascontiguousarray(a))
    if dtype is not None:
        t = t.to(dtype)
    return t.cuda()


def _sub_from_case(eng, c, padded=True, idx_bytes=None):
    nseg = tuple(int(v) for v in c["nseg"])
    if padded:
        from oracle.cells_oracle import padded_as_lists
        ncell = nseg[0] * nseg[1] * nseg[2]
        cells = padded_as_lists(int(c["K"]), c["segments"], ncell)
    else:
        cells = None
    return eng.DeviceSubstrate(c["spheres"], int(c["nstructures"]), tuple(c["L"]), nseg, c["D"], c["T2"], cells=cells,
                               idx_bytes=idx_bytes)


# the fused walk's list forms: per-entry records, 16-bit and 32-bit index lists
LIST_FORMS = [0, 2, 4]


def test_cells_match_oracle(eng):
    z = np.load(__import__("tests._fixtures", fromlist=["GOLDEN"]).GOLDEN / "segments.npz")
    for i in range(int(z["ncase"])):
        sph, L3, nseg = z[f"case{i}_spheres"], tuple(z[f"case{i}_L"]), tuple(int(v) for v in z[f"case{i}_nseg"])
        sub = eng.DeviceSubstrate(sph, 3, L3, nseg, np.full(4, 2.0), np.full(4, 100.0))
        st, ct, it = cells_members(sph, L3, nseg)
        np.testing.assert_array_equal(sub.cell_count.cpu().numpy(), ct)
        np.testing.assert_array_equal(sub.cell_start.cpu().numpy(), st)
        np.testing.assert_array_equal(sub.cell_items.cpu().numpy()[:it.size], it)
        K, seg = sub.padded_segments()
        K_ref, seg_ref = segments_reference(sph, L3, nseg)
        assert K == K_ref == int(z[f"case{i}_K"])
        np.testing.assert_array_equal(seg.cpu().numpy(), seg_ref)


def test_padded_table_full_size(eng):
    """The reference's padded table built on the GPU (nz_segments_fill) for
    the packed workload's 29,628 spheres on 40x40x80 cells (K = 45) against
    the oracle's C restatement of set_segments."""
    from nozomi_b200.substrates import cell_grid
    from nozomi_b200.workloads import packed_workload
    sub = packed_workload()[0]
    nseg = cell_grid(sub.L, 1.0)
    dsub = eng.DeviceSubstrate(sub.spheres(), sub.nstructures, sub.L, nseg, np.full(sub.nstructures + 1, 2.0),
                               np.full(sub.nstructures + 1, 100.0))
    K, seg = dsub.padded_segments()
    assert K == int(oz.cells(sub.spheres(), sub.L, nseg)[1].max())
    np.testing.assert_array_equal(seg.cpu().numpy(), oz.segments(sub.spheres(), sub.L, nseg, K))


@pytest.mark.parametrize("name", NARROW)
def test_plain_narrow_matches_reference(eng, name):
    c = load(name)
    sub = _sub_from_case(eng, c)
    N = int(c["N"])
    x = _dev(c["x0"])
    wk = eng.Walkers.with_counters(x, x.clone(), sig=torch.ones(N, device="cuda"))
    d = eng.philox_draws(int(c["key"]))
    for s in range(int(c["nt"])):
        eng.walk_step(sub, wk, eng.L.MODE_SIG, float(c["dt"]), 0.0, 0.0, s, d)
    np.testing.assert_array_equal(wk.spins.cpu().numpy(), c["spins"])
    np.testing.assert_array_equal(wk.spins0.cpu().numpy(), c["spins0"])
    np.testing.assert_allclose(wk.sig.cpu().numpy(), c["sig"], rtol=2e-6)
    # labels and collision counts against the oracle on the same inputs
    g = oracle_geometry(c)
    spins, spins0 = c["x0"].copy(), c["x0"].copy()
    sig = np.ones(N, np.float32)
    r = oz.walk_f32(g, oz.philox(int(c["key"])), oz.MODE_SIG, spins, spins0, 0, int(c["nt"]), float(c["dt"]), sig=sig)
    np.testing.assert_array_equal(wk.label.cpu().numpy(), r["label"])
    np.testing.assert_array_equal(wk.n_scatter.cpu().numpy(), r["n_scatter"])
    np.testing.assert_array_equal(wk.n_iter.cpu().numpy(), r["n_iter"])
    np.testing.assert_array_equal(wk.flags.cpu().numpy(), r["flags"])


@pytest.mark.parametrize("name", DWI + EDGE)
def test_plain_dwi_matches_reference(eng, name):
    c = load(name)
    sub = _sub_from_case(eng, c)
    N = int(c["N"])
    dirs = dirs_of(c)
    x = _dev(c["x0"].astype(np.float32))
    wk = eng.Walkers.with_counters(x, x.clone(), phase=torch.zeros((dirs.shape[1], N), device="cuda"),
                                   diffdir=_dev(dirs))
    d = eng.philox_draws(int(c["key"]))
    G, Ga = c["G"], c["Garea"]
    for s in range(int(c["nt"])):
        eng.walk_step(sub, wk, eng.L.MODE_PHASE, float(c["dt"]), float(G[s]), float(Ga[s]), s, d)
    np.testing.assert_array_equal(wk.spins.cpu().numpy(), c["spins"])
    np.testing.assert_array_equal(wk.spins0.cpu().numpy(), c["spins0"])
    np.testing.assert_array_equal(wk.phase.cpu().numpy(), c["phase"])


@pytest.mark.parametrize("idx_bytes", LIST_FORMS)
@pytest.mark.parametrize("name", DWI + EDGE + NARROW[:2])
def test_fused_matches_oracle_and_reference(eng, name, idx_bytes):
    """The fused kernel (one launch for all steps, Phi form) against the oracle
    with the same cell lists: positions, spins0, labels and Phi bit-exact; and
    positions against the reference's own outputs.  In every list form."""
    c = load(name)
    sub = _sub_from_case(eng, c, idx_bytes=idx_bytes)
    N = int(c["N"])
    nt = int(c["nt"])
    dt = float(c["dt"])
    G = c["G"] if "G" in c else np.zeros(nt, np.float32)
    Ga = c["Garea"] if "Garea" in c else np.zeros(nt, np.float32)
    x = _dev(c["x0"].astype(np.float32))
    wk = eng.Walkers(x, x.clone(), phi=torch.zeros((6, N), device="cuda"),
                     label=torch.full((N,), -1, dtype=torch.int32, device="cuda"),
                     flags=torch.zeros(N, dtype=torch.int32, device="cuda"), sig=torch.ones(N, device="cuda"))
    st = eng.FusedState.from_walkers(wk)
    mode = eng.L.MODE_PHI | eng.L.MODE_SIG
    eng.walk_fused(sub, st, mode, dt, _dev(G.astype(np.float32)), _dev(Ga.astype(np.float32)), 0, nt,
                   eng.philox_draws(int(c["key"])))
    st.to_walkers(wk)
    g = oracle_geometry(c)
    spins, spins0 = c["x0"].astype(np.float32).copy(), c["x0"].astype(np.float32).copy()
    phi = np.zeros((6, N), np.float32)
    sig = np.ones(N, np.float32)
    r = oz.walk_f32(g, oz.philox(int(c["key"])), oz.MODE_PHI | oz.MODE_SIG, spins, spins0, 0, nt, dt, G=G,
                    Garea=Ga, phi=phi, sig=sig)
    np.testing.assert_array_equal(wk.spins.cpu().numpy(), spins)
    np.testing.assert_array_equal(wk.spins.cpu().numpy(), c["spins"])
    np.testing.assert_array_equal(wk.spins0.cpu().numpy(), spins0)
    np.testing.assert_array_equal(wk.phi.cpu().numpy(), phi)
    np.testing.assert_array_equal(wk.label.cpu().numpy(), r["label"])
    np.testing.assert_array_equal(wk.flags.cpu().numpy(), r["flags"])
    np.testing.assert_allclose(wk.sig.cpu().numpy(), sig, rtol=2e-6)


@pytest.mark.parametrize("by_label", [False, True])
def test_fused_chunked_and_sorted_equals_single_launch(eng, by_label):
    """Splitting the steps over launches and re-binning walkers between them
    (by cell, or by label and cell) changes nothing: draws are keyed by walker
    id and step."""
    c = load("dwi_c1_cells")
    sub = _sub_from_case(eng, c, padded=False)
    N, nt, dt = int(c["N"]), int(c["nt"]), float(c["dt"])
    G, Ga = _dev(c["G"]), _dev(c["Garea"])
    x = _dev(c["x0"].astype(np.float32))

    def fresh():
        wk = eng.Walkers(x.clone(), x.clone(), phi=torch.zeros((6, N), device="cuda"))
        return eng.FusedState.from_walkers(wk)

    d = eng.philox_draws(99)
    a = fresh()
    eng.walk_fused(sub, a, eng.L.MODE_PHI, dt, G, Ga, 0, nt, d)
    b = fresh()
    tmp = eng.FusedState(N)
    scratch = None
    nl = int(c["nstructures"]) + 1 if by_label else 0
    for s0 in range(0, nt, 700):
        scratch = b.sort_into(tmp, sub.grid, 2, scratch, nlabels=nl)
        b, tmp = tmp, b
        eng.walk_fused(sub, b, eng.L.MODE_PHI, dt, G, Ga, s0, min(nt, s0 + 700), d)
    ia = a.walker_ids().cpu().numpy()
    ib = b.walker_ids().cpu().numpy()
    oa, ob = np.argsort(ia), np.argsort(ib)
    for t in ("pos", "org", "phi", "comp"):
        np.testing.assert_array_equal(getattr(a, t).cpu().numpy()[oa], getattr(b, t).cpu().numpy()[ob])


def test_compact_lists_match_oracle(eng):
    """Compact (member-only) cell lists: GPU plain and fused kernels against the
    oracle using the same compact lists."""
    c = load("dwi_overlap")
    sph, L3, nseg = c["spheres"], tuple(c["L"]), tuple(int(v) for v in c["nseg"])
    sub = eng.DeviceSubstrate(sph, int(c["nstructures"]), L3, nseg, c["D"], c["T2"])
    st_, ct, it = cells_members(sph, L3, nseg)
    g = oz.Geometry(sph.astype(np.float32), int(c["nstructures"]), L3, nseg, st_, ct, it, c["D"], c["T2"],
                    dL=tuple(c["dL"]))
    N, nt, dt = int(c["N"]), int(c["nt"]), float(c["dt"])
    dirs = c["dirs"].astype(np.float32)
    x0 = c["x0"].astype(np.float32)
    spins, spins0 = x0.copy(), x0.copy()
    phase = np.zeros((dirs.shape[1], N), np.float32)
    r = oz.walk_f32(g, oz.philox(5), oz.MODE_PHASE, spins, spins0, 0, nt, dt, G=c["G"], Garea=c["Garea"],
                    phase=phase, diffdir=dirs)
    x = _dev(x0)
    wk = eng.Walkers.with_counters(x, x.clone(), phase=torch.zeros((dirs.shape[1], N), device="cuda"),
                                   diffdir=_dev(dirs))
    for s in range(nt):
        eng.walk_step(sub, wk, eng.L.MODE_PHASE, dt, float(c["G"][s]), float(c["Garea"][s]), s, eng.philox_draws(5))
    np.testing.assert_array_equal(wk.spins.cpu().numpy(), spins)
    np.testing.assert_array_equal(wk.phase.cpu().numpy(), phase)
    np.testing.assert_array_equal(wk.n_scatter.cpu().numpy(), r["n_scatter"])
    np.testing.assert_array_equal(wk.label.cpu().numpy(), r["label"])


def test_injected_table_draws(eng):
    """Injected normal tables, exhaustion included (a drained table reads 0)."""
    c = load("narrow_chain_out")
    sub = _sub_from_case(eng, c)
    N, nt = int(c["N"]), 40
    rng = np.random.default_rng(3)
    table = rng.standard_normal((N, nt, 6), dtype=np.float32)  # at most 2 draws per step
    g = oracle_geometry(c)
    spins, spins0 = c["x0"].copy(), c["x0"].copy()
    sig = np.ones(N, np.float32)
    r = oz.walk_f32(g, oz.injected(table), oz.MODE_SIG, spins, spins0, 0, nt, float(c["dt"]), sig=sig)
    assert (r["flags"] & oz.FLAG_DRAWS_EXHAUSTED).any()
    x = _dev(c["x0"])
    wk = eng.Walkers.with_counters(x, x.clone(), sig=torch.ones(N, device="cuda"))
    tab = _dev(table)
    for s in range(nt):
        eng.walk_step(sub, wk, eng.L.MODE_SIG, float(c["dt"]), 0.0, 0.0, s, eng.injected_draws(tab))
    np.testing.assert_array_equal(wk.spins.cpu().numpy(), spins)
    np.testing.assert_array_equal(wk.flags.cpu().numpy(), r["flags"])
    np.testing.assert_array_equal(wk.n_scatter.cpu().numpy(), r["n_scatter"])


def test_seeding_matches_oracle(eng):
    c = load("dwi_overlap")
    sph, L3, nseg = c["spheres"], tuple(c["L"]), tuple(int(v) for v in c["nseg"])
    sub = eng.DeviceSubstrate(sph, 3, L3, nseg, c["D"], c["T2"])
    st_, ct, it = cells_members(sph, L3, nseg)
    g = oz.Geometry(sph.astype(np.float32), 3, L3, nseg, st_, ct, it, c["D"], c["T2"], dL=tuple(c["dL"]))
    for targets in ([0, 1, 2], [3], [1], [0, 1, 2, 3]):
        spins, label = eng.seed(sub, targets, 5000, key=77)
        ref_spins, ref_label, left = oz.seed(g, targets, 5000, key0=77, key1=0, stream=1)
        assert left == 0
        np.testing.assert_array_equal(spins.cpu().numpy(), ref_spins)
        np.testing.assert_array_equal(label.cpu().numpy(), ref_label)


def test_seeding_reports_empty_target(eng):
    sph = np.array([[0.0], [0.0], [0.0], [1e-6], [0.0]])
    sub = eng.DeviceSubstrate(sph, 1, (10.0, 10.0, 10.0), (1, 1, 1), [2.0, 2.0], [100.0, 100.0])
    with pytest.raises(eng.NozomiError):
        eng.seed(sub, [0], 64, key=1, max_rounds=50)


def test_signal_and_moments_match_oracle(eng):
    rng = np.random.default_rng(8)
    N = 20000
    phi = rng.normal(0, 3, (6, N)).astype(np.float32)
    phi[3:] *= 1e-6
    x = _dev(rng.normal(0, 1, (3, N)).astype(np.float32))
    wk = eng.Walkers(x, x.clone(), phi=_dev(phi))
    st = eng.FusedState.from_walkers(wk)
    dirs = rng.standard_normal((3, 7))
    dirs /= np.linalg.norm(dirs, axis=0)
    amps = np.array([0.0, 0.3, 1.0, 2.5])
    out = st.signal(_dev(dirs.astype(np.float32)), _dev(amps.astype(np.float32)))
    S = (out[0] + 1j * out[1]).cpu().numpy() / N
    ref = oz.signal_phi(phi, dirs.astype(np.float32), amps.astype(np.float32))
    np.testing.assert_allclose(S, ref, atol=1e-6)
    s0 = rng.normal(0, 1, (3, N)).astype(np.float32)
    m = torch.zeros(6, dtype=torch.float64, device="cuda")
    eng.moments(x, _dev(s0), m)
    np.testing.assert_allclose(m.cpu().numpy(), oz.moments(x.cpu().numpy(), s0), rtol=1e-10)


@pytest.mark.parametrize("idx_bytes", [0, 2])
@pytest.mark.parametrize("name,margin", [("dwi_c1_cells", 0.5), ("dwi_c1_cells", 0.25), ("dwi_overlap", 0.4),
                                         ("narrow_periodic_in", 0.3), ("dwi_faces", 0.3), ("dwi_faces", 0.6)])
def test_fused_near_lists_match_full_lists(eng, name, margin, idx_bytes):
    """Near lists (smaller margin, used when an iteration's reach fits) give
    the full lists' result bit for bit: the fused walk with near lists against
    the oracle on the full member lists, records and 16-bit index form."""
    c = load(name)
    sph, L3, nseg = c["spheres"], tuple(c["L"]), tuple(int(v) for v in c["nseg"])
    sub = eng.DeviceSubstrate(sph, int(c["nstructures"]), L3, nseg, c["D"], c["T2"], near_margin=margin,
                              idx_bytes=idx_bytes)
    assert sub.near is not None and sub.near[2].numel() < sub.n_items
    st_, ct, it = cells_members(sph, L3, nseg)
    g = oz.Geometry(sph.astype(np.float32), int(c["nstructures"]), L3, nseg, st_, ct, it, c["D"], c["T2"],
                    dL=tuple(c["dL"]))
    N, nt, dt = int(c["N"]), int(c["nt"]), float(c["dt"])
    G = c["G"] if "G" in c else np.zeros(nt, np.float32)
    Ga = c["Garea"] if "Garea" in c else np.zeros(nt, np.float32)
    x0 = c["x0"].astype(np.float32)
    spins, spins0 = x0.copy(), x0.copy()
    phi = np.zeros((6, N), np.float32)
    r = oz.walk_f32(g, oz.philox(17), oz.MODE_PHI, spins, spins0, 0, nt, dt, G=G, Garea=Ga, phi=phi)
    x = _dev(x0)
    wk = eng.Walkers(x, x.clone(), phi=torch.zeros((6, N), device="cuda"),
                     label=torch.full((N,), -1, dtype=torch.int32, device="cuda"),
                     flags=torch.zeros(N, dtype=torch.int32, device="cuda"))
    st = eng.FusedState.from_walkers(wk)
    eng.walk_fused(sub, st, eng.L.MODE_PHI, dt, _dev(G.astype(np.float32)), _dev(Ga.astype(np.float32)), 0, nt,
                   eng.philox_draws(17))
    st.to_walkers(wk)
    np.testing.assert_array_equal(wk.spins.cpu().numpy(), spins)
    np.testing.assert_array_equal(wk.spins0.cpu().numpy(), spins0)
    np.testing.assert_array_equal(wk.phi.cpu().numpy(), phi)
    np.testing.assert_array_equal(wk.label.cpu().numpy(), r["label"])
    np.testing.assert_array_equal(wk.flags.cpu().numpy(), r["flags"])


def test_fused_moments_equal_per_step_moments(eng):
    """Narrow-pulse moments accumulated inside the fused walk (per-CTA FP64
    shared-memory sums of nz_moments' terms) against the plain walk with one
    moment reduction per step (computeDiffusionCoefficientsAndKurtosis's role,
    sim3d_kernel.cu:162-238): identical trajectories, per-step sums equal to
    FP64 summation order.  3001 walkers leave partial warps; 300 steps span
    two launches."""
    from nozomi_b200 import _lib as L
    from nozomi_b200.simulate import device_substrate
    from nozomi_b200.substrates import axon_bundle
    sub = axon_bundle(12, seed=3)
    dsub = device_substrate(sub, D=2.0, cell=0.5, near_margin=0.5)
    N, nt, dt = 3001, 300, 0.005
    x0, lab = eng.seed(dsub, list(range(sub.nstructures + 1)), N, key=99)
    draws = eng.philox_draws(4242)
    # plain: one launch and one moment reduction per step
    wk = eng.Walkers.with_counters(x0.clone(), x0.clone(), sig=torch.ones(N, device="cuda"))
    per_step = torch.zeros((nt, 6), dtype=torch.float64, device="cuda")
    for s in range(nt):
        eng.walk_step(dsub, wk, L.MODE_SIG, dt, 0.0, 0.0, s, draws)
        eng.moments(wk.spins, wk.spins0, per_step[s])
    # fused: moments inside the walk, at most L.MOMENT_STEPS steps per launch
    w2 = eng.Walkers(x0.clone(), x0.clone(), sig=torch.ones(N, device="cuda"), label=lab.clone(),
                     phi=torch.zeros((6, N), device="cuda"))
    st = eng.FusedState.from_walkers(w2)
    fused = torch.zeros((nt, 6), dtype=torch.float64, device="cuda")
    zeros = torch.zeros(nt, device="cuda")
    for s0 in range(0, nt, L.MOMENT_STEPS):
        eng.walk_fused(dsub, st, L.MODE_SIG | L.MODE_MOMENTS, dt, zeros, zeros, s0, min(nt, s0 + L.MOMENT_STEPS),
                       draws, moments=fused)
    out = eng.Walkers(torch.empty((3, N), device="cuda"), torch.empty((3, N), device="cuda"),
                      sig=torch.empty(N, device="cuda"))
    st.to_walkers_by_id(out)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(out.spins.cpu().numpy(), wk.spins.cpu().numpy())
    np.testing.assert_array_equal(out.sig.cpu().numpy(), wk.sig.cpu().numpy())
    np.testing.assert_allclose(fused.cpu().numpy(), per_step.cpu().numpy(), rtol=1e-12, atol=0)
    # the displacement form (nz_walk_fused_moments): every term is nz_moments',
    # so the sums agree to FP64 summation order; any number of steps per call
    w3 = eng.Walkers(x0.clone(), x0.clone(), sig=torch.ones(N, device="cuda"), label=lab.clone(),
                     phi=torch.zeros((6, N), device="cuda"))
    st3 = eng.FusedState.from_walkers(w3)
    disp = torch.zeros((nt, 6), dtype=torch.float64, device="cuda")
    scratch = None
    for s0, s1 in ((0, 7), (7, 300)):
        scratch = eng.walk_fused_moments(dsub, st3, L.MODE_SIG, dt, s0, s1, draws, disp, scratch)
    out3 = eng.Walkers(torch.empty((3, N), device="cuda"), torch.empty((3, N), device="cuda"),
                       sig=torch.empty(N, device="cuda"))
    st3.to_walkers_by_id(out3)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(out3.spins.cpu().numpy(), wk.spins.cpu().numpy())
    np.testing.assert_array_equal(out3.sig.cpu().numpy(), wk.sig.cpu().numpy())
    np.testing.assert_allclose(disp.cpu().numpy(), per_step.cpu().numpy(), rtol=1e-12, atol=0)
    with pytest.raises(eng.NozomiError):  # scratch too small
        L.check(L.load().nz_walk_fused_moments(L.byref(dsub.struct()), L.byref(st3.struct()), 0, 0.005, None, None,
                                               0, 10, L.byref(draws), scratch.data_ptr(), 16,
                                               disp.data_ptr(), torch.cuda.current_stream().cuda_stream),
                "nz_walk_fused_moments")


def test_sort_with_many_bins(eng):
    """Re-binning with more bins than one CTA scans (128,000 bins: the
    multi-CTA scan) and with labels (3 x 128,000 keys): the output is the
    input's walkers, each record intact, in non-decreasing key order."""
    rng = np.random.default_rng(21)
    N = 250_000
    pos = np.stack([rng.uniform(-20, 20, N), rng.uniform(-20, 20, N), rng.uniform(-40, 40, N)]).astype(np.float32)
    lab = rng.integers(0, 3, N).astype(np.int32)
    x = _dev(pos)
    wk = eng.Walkers(x, x + 0.25, phi=_dev(rng.normal(0, 1, (6, N)).astype(np.float32)), label=_dev(lab))
    src = eng.FusedState.from_walkers(wk)
    grid = eng.box_grid((40.0, 40.0, 80.0), (40, 40, 80))

    def canon(st):
        p = st.pos.cpu().numpy()
        ids = st.org.cpu().numpy()[:, 3].view(np.int32)
        ix = np.clip(np.floor((p[:, 0] + 20.0) / 1.0), 0, 39).astype(np.int64)
        iy = np.clip(np.floor((p[:, 1] + 20.0) / 1.0), 0, 39).astype(np.int64)
        iz = np.clip(np.floor((p[:, 2] + 40.0) / 1.0), 0, 79).astype(np.int64)
        cell = (iz * 40 + iy) * 40 + ix
        order = np.argsort(ids)
        rec = np.concatenate([getattr(st, t).cpu().numpy()[order] for t in ("pos", "org", "phi", "comp")], axis=1)
        return cell, p[:, 3].view(np.int32), ids, rec

    _, _, ids0, rec0 = canon(src)
    for nlabels in (0, 3):
        out = eng.FusedState(N)
        src.sort_into(out, grid, 1, nlabels=nlabels)
        torch.cuda.synchronize()
        cell, label, ids, rec = canon(out)
        np.testing.assert_array_equal(np.sort(ids), np.arange(N))
        np.testing.assert_array_equal(rec, rec0)
        key = cell if nlabels == 0 else label.astype(np.int64) * 128000 + cell  # label * bins + bin
        assert np.all(np.diff(key) >= 0)


def test_batch_sort_equals_per_job_sorts(eng):
    """One re-binning pass over three jobs of different grids, walker counts
    and label counts (nz_batch_sort): each job's output is a permutation of
    its own walkers, records intact, in non-decreasing (label, bin) or bin
    order of its own grid, as nz_state_sort_keyed leaves them."""
    import ctypes
    from nozomi_b200 import _lib as L
    from nozomi_b200.batch import _sort_table
    rng = np.random.default_rng(22)
    cases = [((40.0, 40.0, 80.0), (40, 40, 80), 2, 3, 70_001),
             ((12.0, 9.0, 20.0), (12, 9, 20), 4, 0, 5_000),
             ((30.0, 30.0, 30.0), (60, 60, 60), 8, 7, 131_072)]
    jobs, pairs = [], []
    for L3, nseg, coarsen, nl, N in cases:
        pos = np.stack([rng.uniform(-L3[a] / 2, L3[a] / 2, N) for a in range(3)]).astype(np.float32)
        lab = rng.integers(-1, max(nl, 1) + 1, N).astype(np.int32)
        x = _dev(pos)
        wk = eng.Walkers(x, x + 0.5, phi=_dev(rng.normal(0, 1, (6, N)).astype(np.float32)), label=_dev(lab))
        src, dst = eng.FusedState.from_walkers(wk), eng.FusedState(N)
        sub = type("S", (), {"grid": eng.box_grid(L3, nseg), "nstructures": max(nl - 1, 0)})()
        jobs.append((L3, nseg, coarsen, nl, src, dst))
        pairs.append(({"sub": sub}, src, dst))
    # nlabels per job as the table builder would set them (nstructures + 1 when by label)
    table, n, tw, tk = _sort_table(pairs, 1, True)
    raw = bytearray(table.cpu().numpy().tobytes())
    arr = (L.SortJob * n).from_buffer(raw)
    for i, (L3, nseg, coarsen, nl, src, dst) in enumerate(jobs):
        arr[i].coarsen, arr[i].nlabels = coarsen, nl
    tk = 0
    for i, (L3, nseg, coarsen, nl, src, dst) in enumerate(jobs):
        arr[i].key_offset = tk
        tk += int(L.load().nz_sort_job_keys(L.byref(arr[i].grid), coarsen, nl))
    table = torch.from_numpy(np.frombuffer(bytes(raw), dtype=np.uint8).copy()).cuda()
    scratch = torch.empty(int(L.load().nz_batch_sort_scratch_bytes(tw, tk)), dtype=torch.uint8, device="cuda")
    L.check(L.load().nz_batch_sort(ctypes.c_void_p(table.data_ptr()), n, tw, tk, ctypes.c_void_p(scratch.data_ptr()),
                                   scratch.numel(), ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)),
            "nz_batch_sort")
    torch.cuda.synchronize()
    for L3, nseg, coarsen, nl, src, dst in jobs:
        rec = lambda st: np.concatenate([getattr(st, t).cpu().numpy() for t in ("pos", "org", "phi", "comp")], 1)  # noqa: E731
        a, b = rec(src), rec(dst)
        ia, ib = a[:, 7].view(np.int32), b[:, 7].view(np.int32)
        np.testing.assert_array_equal(np.sort(ib), np.arange(src.N))
        np.testing.assert_array_equal(a[np.argsort(ia)], b[np.argsort(ib)])
        p = b[:, :3].astype(np.float32)
        idx = []
        for ax in range(3):
            half, d = np.float32(L3[ax] / 2), np.float32(L3[ax] / nseg[ax])
            c = np.floor((p[:, ax] + half) / d)
            idx.append(np.clip(c, 0, nseg[ax] - 1).astype(np.int64) // coarsen)
        bx, by = -(-nseg[0] // coarsen), -(-nseg[1] // coarsen)
        nbins = bx * by * -(-nseg[2] // coarsen)
        key = (idx[2] * by + idx[1]) * bx + idx[0]
        if nl > 0:
            lab = b[:, 3].view(np.int32).astype(np.int64)
            lab = np.where((lab < 0) | (lab >= nl), nl - 1, lab)
            key = key + lab * nbins
        assert np.all(np.diff(key) >= 0)


@pytest.mark.parametrize("idx_bytes", [2, 4])
def test_index_lists_with_shuffled_sphere_order(eng, idx_bytes):
    """Spheres given out of structure order (a seeded shuffle of the overlap
    fixture's 24 spheres over 3 structures): the index form sorts them into
    records by structure, and the fused walk still equals the oracle on the
    shuffled input bit for bit (positions, Phi, labels, flags)."""
    c = load("dwi_overlap")
    perm = np.random.default_rng(5).permutation(c["spheres"].shape[1])
    sph = c["spheres"][:, perm]
    assert not np.all(np.diff(sph[4]) >= 0)
    L3, nseg = tuple(c["L"]), tuple(int(v) for v in c["nseg"])
    sub = eng.DeviceSubstrate(sph, int(c["nstructures"]), L3, nseg, c["D"], c["T2"], near_margin=0.4,
                              idx_bytes=idx_bytes)
    st_, ct, it = cells_members(sph, L3, nseg)
    g = oz.Geometry(sph.astype(np.float32), int(c["nstructures"]), L3, nseg, st_, ct, it, c["D"], c["T2"],
                    dL=tuple(c["dL"]))
    N, nt, dt = int(c["N"]), int(c["nt"]), float(c["dt"])
    x0 = c["x0"].astype(np.float32)
    spins, spins0, phi = x0.copy(), x0.copy(), np.zeros((6, N), np.float32)
    r = oz.walk_f32(g, oz.philox(23), oz.MODE_PHI, spins, spins0, 0, nt, dt, G=c["G"], Garea=c["Garea"], phi=phi)
    x = _dev(x0)
    wk = eng.Walkers(x, x.clone(), phi=torch.zeros((6, N), device="cuda"),
                     label=torch.full((N,), -1, dtype=torch.int32, device="cuda"),
                     flags=torch.zeros(N, dtype=torch.int32, device="cuda"))
    st = eng.FusedState.from_walkers(wk)
    eng.walk_fused(sub, st, eng.L.MODE_PHI, dt, _dev(c["G"].astype(np.float32)), _dev(c["Garea"].astype(np.float32)),
                   0, nt, eng.philox_draws(23))
    st.to_walkers(wk)
    np.testing.assert_array_equal(wk.spins.cpu().numpy(), spins)
    np.testing.assert_array_equal(wk.phi.cpu().numpy(), phi)
    np.testing.assert_array_equal(wk.label.cpu().numpy(), r["label"])
    np.testing.assert_array_equal(wk.flags.cpu().numpy(), r["flags"])


def test_rounded_near_lists_match_oracle(eng):
    """The near lists' Euclidean test on the device (nz_cells_count_round /
    nz_cells_fill_round) against the numpy restatement, list for list; each
    a subset of the box test's lists with the same margin, and smaller."""
    from oracle.cells_oracle import cells_round
    from nozomi_b200.substrates import axon_bundle, cell_grid
    sub = axon_bundle(25, seed=4)
    sph, L3 = sub.spheres(), sub.L
    nseg = cell_grid(L3, 0.5)
    ns = sub.nstructures
    for margin in (0.3, 0.5):
        d = eng.DeviceSubstrate(sph, ns, L3, nseg, np.full(ns + 1, 2.0), np.full(ns + 1, 100.0), near_margin=margin)
        box = eng.DeviceSubstrate(sph, ns, L3, nseg, np.full(ns + 1, 2.0), np.full(ns + 1, 100.0),
                                  near_margin=margin, near_round=False)
        st, ct, it, n = d.near[0].cpu().numpy(), d.near[1].cpu().numpy(), d.near[2].cpu().numpy(), d.near_n
        rst, rct, rit = cells_round(sph, L3, nseg, margin)
        np.testing.assert_array_equal(ct, rct)
        np.testing.assert_array_equal(st, rst)
        np.testing.assert_array_equal(it[:n], rit)
        bct = box.near[1].cpu().numpy()
        assert np.all(ct <= bct) and ct.sum() < 0.9 * bct.sum()
