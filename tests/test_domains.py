"""Host helpers that build the loop's design / non-design ID lists the way
the reference does (no GPU work)."""
import numpy as np


def test_design_nondesign_ids_is_a_set_difference(gpu):
    # non_design_domain.hpp:9-53: sorted unique non-design IDs, design = the rest
    d, nd = gpu.design_nondesign_ids(20, [7, 3, 3, 19, 0])
    assert nd.tolist() == [0, 3, 7, 19]
    assert d.tolist() == [i for i in range(20) if i not in (0, 3, 7, 19)]


def test_nondesign_boxes_follow_the_sample_function(gpu):
    # opt_macro_mma_nondesign.cpp:247-317: centroid strictly inside a box ->
    # non-design with the box's value; each box adds the elements outside it
    # to the design list
    nx, ny, nz = 10, 4, 2
    one = [(1.0, ((4.0, 6.0), (3.0, 4.0), (0.0, 2.0)))]
    x0, d, nd = gpu.nondesign_boxes(nx, ny, nz, one, 0.35)
    e = np.arange(nx * ny * nz)
    i, j = e % nx, e // nx % ny
    inside = (i >= 4) & (i <= 5) & (j == 3)
    assert nd.tolist() == e[inside].tolist()
    assert d.tolist() == e[~inside].tolist()
    assert np.all(x0[inside] == 1.0) and np.all(x0[~inside] == 0.35)
    # a second, disjoint box: every element is outside one of them
    two = one + [(1e-4, ((0.0, 2.0), (0.0, 1.0), (0.0, 2.0)))]
    x0, d, nd = gpu.nondesign_boxes(nx, ny, nz, two, 0.35)
    assert d.tolist() == e.tolist()
    assert len(nd) == inside.sum() + 2 * 1 * 2
    assert np.all(x0[(i <= 1) & (j == 0)] == 1e-4)
    # no boxes: every element is a design element, no non-design ones
    x0, d, nd = gpu.nondesign_boxes(nx, ny, nz, [], 0.35)
    assert d.tolist() == e.tolist() and nd.size == 0 and np.all(x0 == 0.35)
    # an edge on a centroid is outside (strict inequalities)
    x0, d, nd = gpu.nondesign_boxes(nx, ny, nz, [(1.0, ((4.5, 6.0), (0, 4), (0, 2)))], 0.3)
    assert 4 not in (nd % nx)
