"""CPU: the named bench workloads build the configurations the bench quotes —
grid, boundaries, species order (ambient first, then photoelectrons) and the
conductors' surface nodes and cells."""
import numpy as np
import pytest

from fopis_b200 import config


@pytest.mark.parametrize("name,nodes,boundary,nsp,n_cmat,n_cells", [
    ("periodic32", 32, b"PPPPPP", 2, None, None),
    ("cube64", 65, b"DDDDDD", 2, 386, 8 ** 3),
    ("cube128", 129, b"DDDDDD", 3, 1538, 16 ** 3),
    ("cube128_plain", 129, b"DDDDDD", 2, 1538, 16 ** 3),
    ("craft256", 257, b"DDDDDD", 3, 3586, 32 * 16 * 16 + 48 * 4 * 16),
])
def test_workload_geometry(name, nodes, boundary, nsp, n_cmat, n_cells):
    cfg = config.workload(name)
    p = cfg.params
    assert (p.nx, p.ny, p.nz) == (nodes, nodes, nodes)
    assert bytes(p.boundary[:6]) == boundary
    assert p.nspecies == nsp
    kinds = [s.kind for s in cfg.species]
    assert kinds == sorted(kinds, key=lambda k: k != "ambient")      # ambient first
    if n_cmat is None:
        assert not cfg.objects
        return
    (obj,) = cfg.objects
    assert len(np.asarray(obj.nodes).reshape(-1, 3)) == n_cmat
    assert len(np.asarray(obj.cells).reshape(-1, 3)) == n_cells
    if nsp == 3:
        assert obj.emit_species == 2 and cfg.species[2].kind == "photoelectron"
