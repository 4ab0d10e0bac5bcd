"""Element colouring of T3 meshes (host side, no GPU).

The T3 kernels scatter element contributions one colour at a time without
atomics, which is only race-free if no two elements of a colour share a node.
"""
import numpy as np
import pytest

from phast_b200.t3 import color_elements


def split_quads(nx, ny, rng=None):
    """Triangles of an nx x ny quad grid, each quad split along a (random) diagonal."""
    idx = np.arange((nx + 1) * (ny + 1)).reshape(ny + 1, nx + 1)
    tris = []
    for j in range(ny):
        for i in range(nx):
            a, b, c, d = idx[j, i], idx[j, i + 1], idx[j + 1, i + 1], idx[j + 1, i]
            if rng is not None and rng.random() < 0.5:
                tris += [(a, b, d), (b, c, d)]
            else:
                tris += [(a, b, c), (a, c, d)]
    return np.array(tris, dtype=np.int64), (nx + 1) * (ny + 1)


def check_colouring(elements, n_nodes, colors):
    assert colors.shape == (elements.shape[0],) and colors.min() >= 0
    for k in range(int(colors.max()) + 1):
        nodes = elements[colors == k].reshape(-1)
        assert np.unique(nodes).size == nodes.size, f"colour {k} touches a node twice"


@pytest.mark.parametrize("nx,ny,seed", [(1, 1, None), (7, 5, None), (16, 9, 1), (30, 30, 2)])
def test_colours_never_share_a_node(nx, ny, seed):
    rng = None if seed is None else np.random.default_rng(seed)
    el, nn = split_quads(nx, ny, rng)
    colors = color_elements(el, nn)
    check_colouring(el, nn, colors)
    # a node of a structured triangulation touches at most 8 triangles: greedy needs few colours
    assert int(colors.max()) + 1 <= 12


def test_colouring_is_deterministic_and_handles_shuffled_order():
    rng = np.random.default_rng(5)
    el, nn = split_quads(12, 8, rng)
    perm = rng.permutation(el.shape[0])
    a, b = color_elements(el, nn), color_elements(el, nn)
    assert np.array_equal(a, b)
    check_colouring(el[perm], nn, color_elements(el[perm], nn))


def test_c_abi_rejects_bad_colourings_without_gpu():
    """phastb_t3_check_mesh accepts the package's colouring and refuses out-of-range node ids,
    a non-permutation and two elements of one colour sharing a node."""
    import ctypes as C

    from phast_b200 import _lib
    from phast_b200.t3 import color_elements
    nx, ny = 6, 5
    quads = np.array([[j * (nx + 1) + i, j * (nx + 1) + i + 1, (j + 1) * (nx + 1) + i + 1, (j + 1) * (nx + 1) + i]
                      for j in range(ny) for i in range(nx)])
    tri = np.concatenate([quads[:, [0, 1, 2]], quads[:, [0, 2, 3]]]).astype(np.int32)
    n_nodes = (nx + 1) * (ny + 1)
    colors = color_elements(tri, n_nodes)
    order = np.argsort(colors, kind="stable").astype(np.int32)
    nc = int(colors.max()) + 1
    off = np.searchsorted(colors[order], np.arange(nc + 1))
    lib = _lib.load()
    IP = C.POINTER(C.c_int)

    def check(elem, ordr, offs, n=n_nodes):
        e = np.ascontiguousarray(elem.astype(np.int32))
        o = np.ascontiguousarray(ordr.astype(np.int32))
        f = (C.c_int * len(offs))(*[int(v) for v in offs])
        return lib.phastb_t3_check_mesh(n, len(e), e.ctypes.data_as(IP), o.ctypes.data_as(IP), len(offs) - 1, f)

    assert check(tri, order, off) == _lib.OK
    bad = tri.copy()
    bad[3, 1] = n_nodes  # node id out of range
    assert check(bad, order, off) == _lib.ERR_ARG
    dup = order.copy()
    dup[1] = dup[0]  # not a permutation
    assert check(tri, dup, off) == _lib.ERR_ARG
    one = np.array([0, len(tri)])  # every element in one colour: neighbours share nodes
    assert check(tri, order, one) == _lib.ERR_ARG
