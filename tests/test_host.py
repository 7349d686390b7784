"""Host-side pieces without a GPU: the analytic primary of singularity
removal against the oracle's restatement, the mesh's cell lookup, and the
receivers' data types."""
import numpy as np
import pytest

from oracle import dc_oracle as O
from simpeg_dc_torch_b200 import DipoleReceiver, PoleReceiver
from simpeg_dc_torch_b200 import synthetic as syn
from simpeg_dc_torch_b200.primary import source_cells, unit_primary


def test_unit_primary_matches_oracle():
    mesh, survey, _ = syn.tiny_2d()
    kys = np.array([0.01, 0.1, 0.7])
    widths = mesh.h_gridded
    poles, radii = [], []
    for src in survey.source_list:
        pl = [(src.location_a, 1.0)]
        if getattr(src, "location_b", None) is not None:
            pl.append((src.location_b, -1.0))
        poles.append(pl)
        radii.append([float(np.sqrt(np.prod(widths[int(mesh.point2index(
            np.asarray(loc, float)[None, :2])[0])]) / np.pi)) for loc, _ in pl])
    u = unit_primary(mesh, survey, kys)
    assert u.shape == (kys.size, mesh.n_nodes, len(survey.source_list))
    assert O.rel(u, O.unit_primary_2d(mesh.nodes, kys, poles, radii)) < 1e-14
    # finite everywhere, the disc mean at the source nodes included
    assert np.isfinite(u).all()
    cells = source_cells(mesh, survey)
    assert cells.shape == (len(survey.source_list),)


def test_point2index_and_cell_widths():
    mesh, _, _ = syn.tiny_2d()
    nx, nz = mesh.shape_cells
    cc = mesh.cell_centers
    # every cell centre lies in its own cell
    assert np.array_equal(mesh.point2index(cc), np.arange(mesh.nC))
    # nodes on the far boundaries fall in the last cells
    far = np.array([[mesh.nodes_x[-1], mesh.nodes_y[-1]]])
    assert mesh.point2index(far)[0] == mesh.nC - 1
    w = mesh.h_gridded
    assert w.shape == (mesh.nC, 2)
    assert np.allclose(w.prod(1), mesh.cell_volumes)


def test_receiver_data_types():
    m = np.array([[0.0, 0.0]])
    n = np.array([[1.0, 0.0]])
    assert DipoleReceiver(m, n).data_type == "volt"
    assert DipoleReceiver(m, n, "apparent_chargeability").data_type == \
        "apparent_chargeability"
    assert PoleReceiver(m, data_type="apparent_chargeability").data_type == \
        "apparent_chargeability"
    with pytest.raises(ValueError):
        DipoleReceiver(m, n, "apparent_resistivity")
