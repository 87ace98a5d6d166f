"""The CPU oracle pinned to the reference's own outputs (``tests/golden/*.npz``).

The fixtures come from the reference's ``flat_tree.py`` and kernel sources
(``tests/golden/make_golden.py``).  Integer outputs (trees, permutations,
interaction lists) must be identical; floating-point outputs match to 1e-13
normwise (the same arithmetic, summed in the same order, is bit-identical; the
grouped CPU walk of the reference adds exact zeros for excluded pairs).
"""

from __future__ import annotations

import numpy as np
import pytest

from conftest import golden, relative

TREE_ARRAYS = ("perm", "node_center", "node_half", "node_start", "node_end", "node_child",
               "node_depth", "levels")


def _assert_tree(tree, data, prefix):
    assert tree.node_count == int(data[f"{prefix}/node_count"])
    for name in TREE_ARRAYS:
        np.testing.assert_array_equal(getattr(tree, name), data[f"{prefix}/{name}"], err_msg=name)


@pytest.mark.parametrize("cloud", ["uniform", "circle", "clustered", "lattice", "coincident"])
def test_build_equals_reference(oracle, cloud):
    data = golden("build")
    pos = data[f"{cloud}/pos"]
    tree = oracle.OracleTree(pos, np.ones(pos.shape[1]), (0.0, 0.0, 1.0), leaf_capacity=6)
    _assert_tree(tree, data, cloud)
    np.testing.assert_array_equal(tree.sorted_pos, pos[:, tree.perm])


def test_build_deep_chain_and_leaf_depth_variants(oracle):
    data = golden("build")
    tree = oracle.OracleTree(data["chain/pos"], [1, 1, -1], (0, 0, 1), leaf_capacity=1)
    _assert_tree(tree, data, "chain")
    assert tree.node_count == 1 + 4 * 48
    for leaf, depth in ((1, 10), (8, 48)):
        key = f"cloud300_l{leaf}_d{depth}"
        pos = data[f"{key}/pos"]
        tree = oracle.OracleTree(pos, np.ones(300), (0, 0, 1), leaf_capacity=leaf,
                                 max_depth=depth)
        _assert_tree(tree, data, key)


def test_build_non_dyadic_root(oracle):
    data = golden("build")
    pos = data["offroot/pos"]
    tree = oracle.OracleTree(pos, np.zeros(pos.shape[1]), tuple(data["offroot/root"]),
                             leaf_capacity=16)
    _assert_tree(tree, data, "offroot")


def test_moments_equal_reference(oracle):
    data = golden("moments")
    pos, charge = data["pos"], data["charge"]
    tree = oracle.OracleTree(pos, charge, (0, 0, 1), leaf_capacity=8)
    _assert_tree(tree, data, "coulomb")
    for name in ("node_q", "node_qabs", "node_p", "node_s"):
        np.testing.assert_array_equal(getattr(tree, name), data[f"coulomb/{name}"], err_msg=name)
    tree = oracle.OracleTree(pos, charge, (0, 0, 1), leaf_capacity=8, kernel="log", order=12)
    for name in ("node_qabs", "moment_re", "moment_im", "node_q", "node_p"):
        np.testing.assert_array_equal(getattr(tree, name), data[f"log/{name}"], err_msg=name)
    for order in (4, 12):
        tree = oracle.OracleTree(pos, charge, (0, 0, 1), leaf_capacity=8, order=order)
        np.testing.assert_array_equal(tree.cartesian_moments(), data[f"cart{order}/moments"])


def test_cartesian_tables_equal_reference(oracle):
    data = golden("tables")
    for order in (4, 8, 12):
        tables = oracle.cart_tables(order)
        for name, value in tables.items():
            np.testing.assert_array_equal(value, data[f"p{order}/{name}"], err_msg=name)


@pytest.mark.parametrize("kernel", ["coulomb", "log"])
@pytest.mark.parametrize("eps", [0.0, 0.01])
def test_direct_field_equals_reference(oracle, kernel, eps):
    data = golden("direct")
    phi, field = oracle.direct_field(data["targets"], data["pos"], data["charge"],
                                     softening=eps, exclude=data["exclude"], kernel=kernel)
    np.testing.assert_array_equal(phi, data[f"{kernel}/eps{eps}/phi"])
    np.testing.assert_array_equal(field, data[f"{kernel}/eps{eps}/field"])


@pytest.mark.parametrize("kernel", ["coulomb", "log"])
@pytest.mark.parametrize("leaf", [1, 8])
@pytest.mark.parametrize("theta", [0.0, 0.5, 1.2])
def test_walk_equals_reference(oracle, kernel, leaf, theta):
    data = golden("evaluate")
    pos, charge = data["cloud/pos"], data["cloud/charge"]
    depth = 10 if leaf == 1 else 48
    tree = oracle.OracleTree(pos, charge, (0, 0, 1), leaf_capacity=leaf, max_depth=depth,
                             kernel=kernel)
    phi, field = tree.evaluate(pos, exclude=np.arange(pos.shape[1]), theta=theta,
                               softening=0.01)
    key = f"cloud/{kernel}/l{leaf}/t{theta}"
    assert relative(phi, data[f"{key}/phi"]) <= 1e-13
    assert relative(field, data[f"{key}/field"]) <= 1e-13


def test_walk_config1_and_probes(oracle):
    data = golden("evaluate")
    pos, charge = data["config1/pos"], data["config1/charge"]
    tree = oracle.OracleTree(pos, charge, (0, 0, 1))
    ex = np.arange(pos.shape[1])
    phi, field = tree.evaluate(pos, exclude=ex, theta=0.5, softening=1e-3)
    assert relative(phi, data["config1/phi"]) <= 1e-13
    assert relative(field, data["config1/field"]) <= 1e-13
    dphi, dfield = oracle.direct_field(pos, pos, charge, softening=1e-3, exclude=ex)
    np.testing.assert_array_equal(dphi, data["config1/direct_phi"])
    np.testing.assert_array_equal(dfield, data["config1/direct_field"])
    pos, q, probes = data["probes/pos"], data["probes/charge"], data["probes/targets"]
    tree = oracle.OracleTree(pos, q, (0, 0, 1), kernel="log", order=10)
    for potential in (True, False):
        phi, field = tree.evaluate(probes, theta=0.6, potential=potential)
        assert relative(field, data[f"probes/log/pot{int(potential)}/field"]) <= 1e-13
        if potential:
            assert relative(phi, data["probes/log/pot1/phi"]) <= 1e-13
        else:
            assert not np.any(phi) and not np.any(data["probes/log/pot0/phi"])
    tree = oracle.OracleTree(pos, q, (0, 0, 1))
    phi, field = tree.evaluate(probes, theta=0.6, softening=0.002)
    assert relative(phi, data["probes/coulomb/phi"]) <= 1e-13
    assert relative(field, data["probes/coulomb/field"]) <= 1e-13


def test_log_fmm_equals_reference(oracle):
    data = golden("fmm")
    pos, q = data["log/pos"], data["log/charge"]
    tree = oracle.OracleTree(pos, q, (0, 0, 1), kernel="log", order=12)
    phi, field = tree.fmm(theta=0.5)
    m2l, p2p = tree.lists(0.5)
    np.testing.assert_array_equal(m2l, data["log/m2l"])
    np.testing.assert_array_equal(p2p, data["log/p2p"])
    rows, partners = tree.m2l_rows(m2l)
    np.testing.assert_array_equal(rows, data["log/m2l_rows"])
    np.testing.assert_array_equal(partners[: 2 * len(m2l)], data["log/m2l_partners"])
    np.testing.assert_array_equal(phi, data["log/phi"])
    np.testing.assert_array_equal(field, data["log/field"])
    phi, field = tree.fmm(theta=0.5, softening=0.005, potential=False)
    np.testing.assert_array_equal(phi, data["log/eps/phi"])
    np.testing.assert_array_equal(field, data["log/eps/field"])
    tree = oracle.OracleTree(pos, q, (0, 0, 1), kernel="log", order=12, symmetric=True)
    phi, field = tree.fmm(theta=0.4)
    np.testing.assert_array_equal(phi, data["log/sym/phi"])
    np.testing.assert_array_equal(field, data["log/sym/field"])
    tree = oracle.OracleTree(pos, q, (0, 0, 1), kernel="log", order=8, leaf_capacity=1)
    phi, field = tree.fmm(theta=0.6)
    np.testing.assert_array_equal(phi, data["log/leaf1/phi"])
    np.testing.assert_array_equal(field, data["log/leaf1/field"])


@pytest.mark.parametrize("order", [4, 8, 12])
def test_coulomb_fmm_equals_reference(oracle, order):
    data = golden("fmm")
    pos, q = data["coulomb/pos"], data["coulomb/charge"]
    eps = float(data[f"coulomb/p{order}/eps"])
    tree = oracle.OracleTree(pos, q, (0, 0, 1), order=order, leaf_capacity=16)
    phi, field = tree.fmm(theta=0.5, softening=eps)
    np.testing.assert_array_equal(phi, data[f"coulomb/p{order}/phi"])
    np.testing.assert_array_equal(field, data[f"coulomb/p{order}/field"])


@pytest.mark.parametrize("kernel", ["coulomb", "log"])
def test_fmm_at_equals_reference(oracle, kernel):
    data = golden("fmm_at")
    order = 8 if kernel == "coulomb" else 16
    eps = 0.01 if kernel == "coulomb" else 0.0
    tree = oracle.OracleTree(data["pos"], data["charge"], (0, 0, 1), kernel=kernel,
                             order=order, leaf_capacity=16)
    targets = data["targets"]
    ttree = tree.target_tree(targets, 16)
    _assert_tree(ttree, data, f"{kernel}/target_tree")
    (m2l_rows, m2l_p, n_m2l), (p2p_rows, p2p_p, n_p2p) = tree.dual_lists(ttree, 0.5)
    np.testing.assert_array_equal(m2l_rows, data[f"{kernel}/m2l_rows"])
    np.testing.assert_array_equal(m2l_p[:n_m2l], data[f"{kernel}/m2l_partners"])
    np.testing.assert_array_equal(p2p_rows, data[f"{kernel}/p2p_rows"])
    np.testing.assert_array_equal(p2p_p[:n_p2p], data[f"{kernel}/p2p_partners"])
    phi, field = tree.fmm_at(targets, exclude=data["exclude"], theta=0.5, softening=eps)
    np.testing.assert_array_equal(phi, data[f"{kernel}/phi"])
    np.testing.assert_array_equal(field, data[f"{kernel}/field"])


def test_pair_energy_equals_reference(oracle):
    data = golden("energy")
    energy = oracle.pair_energy(data["pos"], data["charge"], 0.01)
    assert energy == pytest.approx(float(data["energy"][0]), rel=1e-13)
