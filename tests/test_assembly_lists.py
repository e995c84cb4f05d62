"""Bus-to-element lists of the device Sbus assembly (CPU): CSR over buses, element order kept
within a bus (the reference adds injections in element order, GridModel.cpp:701-716)."""
import numpy as np

from lightsim2grid_b200.assembly import _bus_lists


def test_bus_lists_keep_element_order():
    buses = np.array([3, 0, 3, 2, 0, 3])
    ptr, ids = _bus_lists(buses, 5)
    assert ptr.tolist() == [0, 2, 2, 3, 6, 6]
    assert ids[ptr[0]:ptr[1]].tolist() == [1, 4]
    assert ids[ptr[3]:ptr[4]].tolist() == [0, 2, 5]
    assert ids[ptr[2]:ptr[3]].tolist() == [3]
