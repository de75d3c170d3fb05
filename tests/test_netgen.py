"""The numpy network writer (cicy_geom_b200.netgen) against the library's generator.

The benchmark's reference arm writes its network files with netgen so the
upstream process never loads libcicy_b200.so; both arms must still run the very
same network, so the files must be byte-identical."""
import filecmp
import os
import tempfile

import pytest

from cicy_geom_b200 import netgen
from cicy_geom_b200.network import NetworkConfig, generate_cnt_network, write_read_network_files


@pytest.mark.parametrize("side,n,seed", [(2.0, 400, 1), (1.6, 700, 7), (3.0, 1500, 2_000_000)])
def test_netgen_files_are_byte_identical_to_the_library_generator(side, n, seed):
    cfg = NetworkConfig(side=side, n_cnts=n, seed=seed, tolerance=1e-8, tolerance_unit=1e-12)
    with tempfile.TemporaryDirectory() as a, tempfile.TemporaryDirectory() as b:
        write_read_network_files(a, generate_cnt_network(cfg), cfg)
        netgen.write_network_files(b, cfg)
        for f in ("cnt_struct.dat", "cnt_coordinates.dat", "sample_geom.csv", "input.dat"):
            assert filecmp.cmp(os.path.join(a, f), os.path.join(b, f), shallow=False), f


def test_netgen_does_not_load_the_library():
    import subprocess
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    code = ("import sys, tempfile; sys.path.insert(0, %r)\n"
            "from cicy_geom_b200 import netgen\nfrom cicy_geom_b200.network import NetworkConfig\n"
            "d = tempfile.mkdtemp(); netgen.write_network_files(d, NetworkConfig(side=1.0, n_cnts=50, seed=3))\n"
            "maps = open('/proc/self/maps').read()\nprint('libcicy_b200' in maps)\n") % root
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, check=True).stdout.strip()
    assert out == "False"
