"""CLI and configuration (host logic on CPU; one end-to-end run on the GPU)."""
import json
import pickle

import numpy as np
import pytest

from nozomi_b200 import config as cfg
from nozomi_b200.cli.main import parser, substrate_files
from nozomi_b200 import substrates as sb


def test_config_merge_keeps_file_values_for_unset_args():
    c = cfg.load_config_file(cfg.SIM_CONFIG_FILE)
    m = cfg.merge(c, {"nseg": None, "sim_time": 5.0})
    assert m["nseg"] == c["nseg"] and m["sim_time"] == 5.0


def test_parser_subcommands():
    a = parser().parse_args(["simulation", "--substrates", "x", "--sim_time", "2", "--nseg", "3"])
    assert a.command == "simulation" and a.sim_time == 2.0 and a.nseg == 3
    g = parser().parse_args(["gradient_simulation", "--substrates", "x"])
    assert g.config.endswith("pgse_sim_params.json")


def _write_substrate(tmp_path):
    """Two straight fibres in the reference's pickle format (last sphere of a
    fibre at z == L/2)."""
    L = 10.0
    rows = []
    for fid, (x, y) in enumerate([(-2.0, 0.0), (2.5, 1.0)]):
        for z in np.linspace(-L / 2 + 0.3, L / 2, 30):
            rows.append([x, y, z, 1.0, fid])
    d = tmp_path / "exp" / "run1" / "data"
    d.mkdir(parents=True)
    sb.save_pickle(d / "sub.pkl", np.array(rows), L)
    return tmp_path / "exp", L


def test_substrate_walk_and_ingestion(tmp_path):
    root, L = _write_substrate(tmp_path)
    files = substrate_files(str(root))
    assert len(files) == 1
    s = sb.from_pickle(files[0])
    assert s.nstructures == 2
    assert all(f.shape[0] == 30 + 50 for f in s.fibers)  # z pads of 25 + 25 spheres


@pytest.mark.gpu
def test_cli_end_to_end(tmp_path):
    from nozomi_b200.cli.main import main
    root, L = _write_substrate(tmp_path)
    conf = tmp_path / "sim.json"
    conf.write_text(json.dumps({"time_step": 0.002, "num_spins": 20000, "D0_intra": 2.0, "D0_extra": 2.0,
                                "nseg": 2, "sim_time": 1.0}))
    assert main(["simulation", "--substrates", str(root), "--config", str(conf), "--compartment", "intra"]) == 0
    out = list((root / "run1" / "sim" / "ADCdata").glob("diffcoeff_intra_*spins_sub_*.pkl"))
    data = pickle.load(open([p for p in out if "kurtosis" not in p.name][0], "rb"))
    assert data.shape == (500, 4)
    # row k: D after step k + 1, at t = (k + 1) dt (aligned, unlike the reference's shifted column)
    np.testing.assert_allclose(data[:, 3], 0.002 * np.arange(1, 501), rtol=1e-12)
    rec = json.loads(next((root / "run1" / "sim" / "ADCdata").glob("*.json")).read_text())
    assert rec["num_spins"] == 20000 and rec["steps"] == 500 and rec["walker_steps_per_s"] > 0
    # fibres along z: free along z, restricted across
    assert 1.6 < data[-1, 2] < 2.4 and data[-1, 0] < 1.0
    g = tmp_path / "g.json"
    g.write_text(json.dumps({"time_step": 0.01, "num_spins": 5000, "D0_intra": 2.0, "D0_extra": 2.0, "nseg": 2,
                             "sim_time": 30.0, "gradient": {"type": "PGSE", "direction": [[1, 0, 0], [0, 0, 1]],
                                                            "big_delta": 20.0, "little_delta": 10.0}}))
    assert main(["gradient_simulation", "--substrates", str(root), "--config", str(g)]) == 0
    res = pickle.load(open(next((root / "run1" / "sim" / "DWIdata").glob("*.pkl")), "rb"))
    assert res["phase"].shape == (2, 5000)
    S = res["signal"].real
    assert S[0, 0] == pytest.approx(1.0) and S[1, -1] < S[0, -1]  # along the fibres attenuates more


def test_ingestion_matches_reference_driver(tmp_path):
    """Substrate ingestion against the reference's own code
    (tests/golden/ingestion.npz, made by make_golden.py: the pickle read by
    import_array_geometry_full_path, split at z == L/2, z-padded by
    createBoundaryZ), on fibres that continue through the z face as another
    fibre, as themselves, or not at all: every sphere, bit for bit."""
    from tests._fixtures import GOLDEN
    z = np.load(GOLDEN / "ingestion.npz")
    A, L = z["matrix"], float(z["L"])
    ref = np.split(z["fibres"], np.cumsum(z["lengths"])[:-1])
    mine = sb.bound_z(sb.split_fibers(A.copy(), L), L)
    assert len(mine) == len(ref)
    for a, b in zip(mine, ref):
        np.testing.assert_array_equal(a, b)
    path = tmp_path / "s.pkl"
    sb.save_pickle(path, A, L)
    s = sb.from_pickle(path)
    assert s.L == (L, L, L) and s.nstructures == len(ref)
    for a, b in zip(s.fibers, ref):
        np.testing.assert_array_equal(a, b[:, :4])


def test_run_record(tmp_path):
    from nozomi_b200.cli.simulation_main import write_run_record
    p = tmp_path / "r.json"
    rec = write_run_record(p, num_spins=1000, steps=500, sim_time_s=0.25, table_time_s=0.1, compartment="intra",
                           D_final=[1.0, 2.0, 3.0])
    assert rec["walker_steps_per_s"] == pytest.approx(2e6)
    assert json.loads(p.read_text()) == rec
    assert write_run_record(tmp_path / "z.json", num_spins=1, steps=1, sim_time_s=0.0)["walker_steps_per_s"] is None
