"""Helpers shared by the GPU tests."""
import numpy as np

FIELDS = ("h0", "qx0", "qy0", "z0", "h1x", "qx1x", "qy1x", "z1x", "h1y", "qx1y", "qy1y", "z1y")


def rel_err(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    if a.size == 0:
        return 0.0
    return float(np.max(np.abs(a - b) / np.maximum(1.0, np.abs(b))))


def assert_same_topology(mine: dict, ref: dict, what: str):
    np.testing.assert_array_equal(mine["act"], ref["act"], err_msg=f"{what}: leaf hierarchy indices")
    np.testing.assert_array_equal(mine["lvl"], ref["lvl"], err_msg=f"{what}: leaf levels")
    np.testing.assert_array_equal(mine["nb_ids"], ref["nb_ids"], err_msg=f"{what}: neighbour ids")
    if ref.get("nb_lvls") is not None:
        np.testing.assert_array_equal(mine["nb_lvls"], ref["nb_lvls"], err_msg=f"{what}: neighbour levels")
