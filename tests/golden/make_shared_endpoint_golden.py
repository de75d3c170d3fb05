"""Golden values for a Monte-Carlo realisation whose window trimming leaves two
CNT segments sharing an end point on a face that is not prescribed in the
real-resistor pass (side 3.39 um, 12,216 CNTs, seed 3,000,057).

Runs oracle/_ref/ref_dump (the upstream sources compiled by oracle/Makefile) on
the network the project's generator writes, and stores the upstream resistance
and system sizes in tests/golden/mc_3000057.json.

  python tests/golden/make_shared_endpoint_golden.py
"""
import json
import os
import subprocess
import sys
import tempfile

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from cicy_geom_b200 import batch as BT  # noqa: E402
from cicy_geom_b200.network import generate_cnt_network, write_read_network_files  # noqa: E402
from oracle.dumpio import read_dump  # noqa: E402

SEED = 3_000_057


def config():
    return [c for c in BT.monte_carlo_configs(64) if c.seed == SEED][0]


def main():
    cfg = config()
    with tempfile.TemporaryDirectory() as d:
        write_read_network_files(d, generate_cnt_network(cfg), cfg)
        subprocess.run([os.path.join(ROOT, "oracle", "_ref", "ref_dump"), "dump", d, d + "/dump.bin"], check=True, capture_output=True)
        z = read_dump(d + "/dump.bin")
    out = {"seed": SEED, "side": cfg.side, "n_cnts": cfg.n_cnts, "tolerance": cfg.tolerance,
           "resistances": [float(x) for x in z["resistances"]],
           "unit_nodes": [int(x) for x in z["c0_u_nodes"]], "real_nodes": [int(x) for x in z["c0_d0_nodes"]]}
    with open(os.path.join(ROOT, "tests", "golden", "mc_3000057.json"), "w") as f:
        json.dump(out, f, indent=1)
    print(out)


if __name__ == "__main__":
    main()
