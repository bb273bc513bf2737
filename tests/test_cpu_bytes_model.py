"""The algorithmic-bytes model (the numerator of the reported roofline).

Per-particle bytes of one substep at 3 iterations: water 1,640 B, snow 3,232 B, boundary
196 B; the density + lambda launch of the 154k-particle scene (5,888 water, 147,928 snow,
52,016 boundary) moves 56 B per particle of all three sets.
"""
from snowsimulation_b200 import bytes_model as bm

NW, NS, NB = 5888, 147928, 52016


def test_per_particle_substep():
    assert bm.per_particle_substep(3) == (1640, 3232, 196)


def test_substep_total_config1():
    total = bm.substep_bytes(NW, NS, NB, 3)
    assert total == NW * 1640 + NS * 3232 + NB * 196
    # about 0.488 GB of water and snow traffic plus the boundary term
    assert abs((NW * 1640 + NS * 3232) / 1e9 - 0.488) < 0.001


def test_density_lambda_launch():
    kb = bm.kernel_bytes("k_density", NW, NS, NB) + bm.PASS["L"] * (NW + NS + NB)
    assert kb == 56 * (NW + NS + NB) == 11526592


def test_one_entry_per_pass_kernel():
    # each stage's bytes belong to the kernel that runs it: contact and interlink are
    # separate launches
    assert bm.kernel_bytes("k_dem_corr", NW, NS, NB) == bm.PASS["X"] * NS
    assert (bm.kernel_bytes("k_link_terms", NW, NS, NB) + bm.kernel_bytes("k_link_sum", NW, NS, NB)
            == bm.PASS["I"] * NS)
    assert bm.kernel_bytes("k_not_a_kernel", NW, NS, NB) is None
