"""Host side of the learned guess on CPU: the node graph the CUDA kernels walk and
the parameter layout agree with the numpy oracle of the network."""
import numpy as np
import pytest

from adh_kraken_b200 import learned
from adh_kraken_b200.mesh import beach_case, small_delaunay_case
from oracle import gnn_oracle


@pytest.mark.parametrize("which", ["wetdry", "beach"])
def test_graph_matches_oracle(which):
    c = small_delaunay_case(n=12, seed=5) if which == "wetdry" else beach_case(nx=60, ny=15, nsteps=1)
    g1 = learned.build_graph(c.xyz[:, :2], c.tri)
    g2 = gnn_oracle.graph_arrays(c.xyz[:, :2], c.tri)
    for k in ("indptr", "nbr", "rev"):
        assert np.array_equal(np.asarray(g1[k]), np.asarray(g2[k])), k
    for k in ("wx", "wy", "inv_deg", "swx", "swy"):
        assert np.allclose(np.asarray(g1[k]), np.asarray(g2[k]), rtol=1e-15, atol=0), k
    assert g1["L"] == g2["L"]
    n = c.nnodes
    nbr, rev, ip = np.asarray(g1["nbr"]), np.asarray(g1["rev"]), np.asarray(g1["indptr"])
    row = np.repeat(np.arange(n), np.diff(ip))
    assert np.array_equal(nbr[rev], row) and np.array_equal(row[rev], nbr)     # rev is the reverse edge
    assert not np.any(nbr == row)                                              # no self loops


def test_parameter_layout_matches_oracle():
    offs, total = gnn_oracle.offsets()
    layout, ltotal = learned.param_layout()
    assert ltotal == total
    assert [(o, i, j) for o, i, j in layout] == offs
