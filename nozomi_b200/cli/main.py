"""Command-line entry (the reference's simulation_toolkit/cli/main.py:94-177):

    python -m nozomi_b200.cli.main simulation --substrates DIR [--sim_time T] [--compartment intra|extra] [--nseg N]
    python -m nozomi_b200.cli.main gradient_simulation --substrates DIR [--config FILE] ...

Walks DIR/*/data/* like the reference (cli/main.py:35-76) and runs one driver
per substrate file; saves the merged configuration next to the substrates.
Substrate generation (``substrate``) is a separate product and not part of
this package.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
from datetime import datetime

from .. import config as cfg


def substrate_files(main_folder):
    if not os.path.isdir(main_folder):
        raise SystemExit(f"Error: {main_folder} is not a valid directory")
    out = []
    for sub in sorted(os.listdir(main_folder)):
        data = os.path.join(main_folder, sub, "data")
        if os.path.isdir(data):
            out += [os.path.join(data, f) for f in sorted(os.listdir(data)) if os.path.isfile(os.path.join(data, f))]
    return out


def parser():
    p = argparse.ArgumentParser(description="nozomi_b200 simulation toolkit")
    sp = p.add_subparsers(dest="command")
    sim = sp.add_parser("simulation", help="narrow-pulse D(t) simulations")
    sim.add_argument("--substrates", type=str, required=True)
    sim.add_argument("--sim_time", type=float)
    sim.add_argument("--compartment", type=str)
    sim.add_argument("--nseg", type=int)
    sim.add_argument("--num_spins", type=int)
    sim.add_argument("--time_step", type=float)
    sim.add_argument("--config", type=str, default=str(cfg.SIM_CONFIG_FILE))
    g = sp.add_parser("gradient_simulation", help="PGSE / OGSE phase and signal simulations")
    g.add_argument("--substrates", type=str, required=True)
    g.add_argument("--sim_time", type=float)
    g.add_argument("--nseg", type=int)
    g.add_argument("--compartment", type=str)
    g.add_argument("--num_spins", type=int)
    g.add_argument("--time_step", type=float)
    g.add_argument("--config", type=str, default=str(cfg.PGSE_CONFIG_FILE))
    sp.add_parser("substrate", help="not part of this package")
    return p


def main(argv=None):
    args = parser().parse_args(argv)
    if not args.command:
        parser().print_help()
        return 0
    if args.command == "substrate":
        print("substrate generation is not part of nozomi_b200; use the reference toolkit's generator", file=sys.stderr)
        return 2
    config = cfg.merge(cfg.load_config_file(args.config), {k: v for k, v in vars(args).items() if k != "config"})
    if args.command == "simulation":
        from .simulation_main import simulation_main as run
    else:
        from .gradient_simulation_main import simulation_gradient_main as run
    outputs = [run(config, f) for f in substrate_files(args.substrates)]
    stamp = datetime.now().strftime("%Y-%m-%d_%H-%M")
    with open(os.path.join(args.substrates, f"{stamp}_{os.path.basename(args.config)}"), "w") as f:
        json.dump(config, f, indent=4)
    return 0 if outputs else 1


if __name__ == "__main__":
    sys.exit(main())
