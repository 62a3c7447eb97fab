"""The benchmark's workloads are the configurations they are named after: interior fluid
cells of config 1 (64^3 Taylor-Green), config 2 (128^3 mixing layer between a characteristic
inflow and outflow) and config 3 (the 512 x 8 x 8 reacting channel), the bounded CPU slab of
config 2 for the reference's timing, and the byte counts the roofline divides by."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


class Args:
    def __init__(self, workload, N, chem="ref", precision="fp64"):
        self.workload, self.N, self.chem, self.precision = workload, N, chem, precision


def test_config_1_is_64_cubed():
    cells, prm = bench.workload(64)
    assert bench.fluid_cells(cells) == 64 ** 3


def test_config_2_is_128_cubed_with_characteristic_ends():
    m, mix, sp = bench.mc_workload(Args("inflow", 128))
    assert bench.fluid_cells(mix) == 128 ** 3
    assert len(sp) == 9
    t = mix["type"]
    assert (t[0] == 7).all() and (t[-1] == 8).all()      # TYPE_I_C inflow, TYPE_O_C outflow in x
    assert not bench.mc_reaction(Args("inflow", 128))


def test_config_3_is_the_512_by_8_by_8_reacting_channel():
    m, mix, sp = bench.mc_workload(Args("flame", 128, chem="rosenbrock", precision="fp32"))
    assert mix.shape == (514, 10, 10)
    assert bench.fluid_cells(mix) == 512 * 8 * 8
    assert bench.mc_reaction(Args("flame", 128))
    name = bench.mc_workload_name(Args("flame", 128, "rosenbrock", "fp32"), "512x8x8")
    assert name.startswith("flame128_mc9_fp32_ros2") and "512x8x8" in name


def test_roofline_bytes_per_cell():
    assert bench.mc_bytes("k_mc_relax", 8) == 2 * 270 * 8 + 84 * 8
    assert bench.mc_bytes("k_mc_relax", 4, reaction=True) == 2 * 270 * 4 + 93 * 8
    assert bench.mc_bytes("k_mc_gather", 8) == 270 * 8 + 91 * 8
    assert bench.mc_bytes("k_mc_solve", 8) == (91 + 21 + 36 + 88) * 8
    assert bench.whole_job_mlups(4, 2 ** 21, 100, 2.0) == 4 * 2 ** 21 * 100 / 2.0 / 1e6
