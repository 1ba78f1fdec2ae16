"""Configuration: JSON files merged with command-line arguments.

Keys and defaults follow the reference's experiment/setup/simulation/*.json
(time_step, num_spins, D0_intra, D0_extra, nseg; sim_time; gradient) and
simulation_toolkit/config.py:13-18.  Unlike the reference (cli/main.py:151),
command-line arguments that were not given do not overwrite file values with
None.
"""
from __future__ import annotations

import json
from pathlib import Path

CONFIG_DIR = Path(__file__).resolve().parent / "configs"
SIM_CONFIG_FILE = CONFIG_DIR / "default-sim.json"
PGSE_CONFIG_FILE = CONFIG_DIR / "pgse_sim_params.json"


def load_config_file(path) -> dict:
    with open(path, "r") as f:
        return json.load(f)


def merge(config: dict, cli_args: dict) -> dict:
    out = dict(config)
    out.update({k: v for k, v in cli_args.items() if v is not None})
    return out
