"""DC surveys: current sources and potential receivers.

Mirrors the attributes of SimPEG's `resistivity.sources`, `.receivers` and
`.survey.Survey` that the engines read (`source_list`, `receiver_list`,
`location_a/b`, `locations_m/n`, `current`, `nD`), so a SimPEG survey object
can be used in place of these classes.

Nodal source term (SimPEG `BaseSrc.eval`, EB formulation): the current
electrode(s) enter the right-hand side through the node interpolation matrix,
`q = I (P_A - P_B)`, with B absent for a pole.  Receivers read
`P = P_M - P_N` (dipole) or `P_M` (pole).  Data type "volt"; a receiver
of an induced-polarization survey may say "apparent_chargeability" instead,
which the DC engines read as volts and the IP engines (`ip.py`) scale by the
background datum, as SimPEG's `BaseIPSimulation._scale` does.
"""
from __future__ import annotations

import numpy as np


_DATA_TYPES = ("volt", "apparent_chargeability")


class _Receiver:
    data_type = "volt"

    def _set_type(self, data_type):
        if data_type not in _DATA_TYPES:
            raise ValueError(f"data_type must be one of {_DATA_TYPES}")
        self.data_type = data_type

    @property
    def nD(self):
        return int(np.atleast_2d(self.locations_m).shape[0])


class DipoleReceiver(_Receiver):
    def __init__(self, locations_m, locations_n, data_type="volt"):
        self._set_type(data_type)
        self.locations_m = np.atleast_2d(np.asarray(locations_m, float))
        self.locations_n = np.atleast_2d(np.asarray(locations_n, float))
        if self.locations_m.shape != self.locations_n.shape:
            raise ValueError("M and N locations must have the same shape")

    def getP(self, mesh, projected_grid="N"):
        return (mesh.get_interpolation_matrix(self.locations_m, "N")
                - mesh.get_interpolation_matrix(self.locations_n, "N")).tocsr()


class PoleReceiver(_Receiver):
    def __init__(self, locations, data_type="volt"):
        self._set_type(data_type)
        self.locations_m = np.atleast_2d(np.asarray(locations, float))
        self.locations_n = None

    @property
    def locations(self):
        return self.locations_m

    def getP(self, mesh, projected_grid="N"):
        return mesh.get_interpolation_matrix(self.locations_m, "N").tocsr()


class DipoleSource:
    def __init__(self, receiver_list, location_a, location_b, current=1.0):
        self.receiver_list = list(receiver_list)
        self.location_a = np.asarray(location_a, float)
        self.location_b = np.asarray(location_b, float)
        self.current = float(current)

    def eval_nodal(self, mesh):
        P = mesh.get_interpolation_matrix(
            np.vstack([self.location_a, self.location_b]), "N").toarray()
        return self.current * (P[0] - P[1])


class PoleSource:
    def __init__(self, receiver_list, location, current=1.0):
        self.receiver_list = list(receiver_list)
        self.location_a = np.asarray(location, float)
        self.location_b = None
        self.current = float(current)

    @property
    def location(self):
        return self.location_a

    def eval_nodal(self, mesh):
        P = mesh.get_interpolation_matrix(
            np.atleast_2d(self.location_a), "N").toarray()
        return self.current * P[0]


class Survey:
    def __init__(self, source_list):
        self.source_list = list(source_list)

    @property
    def nD(self):
        return int(sum(rx.nD for src in self.source_list
                       for rx in src.receiver_list))

    @property
    def nSrc(self):
        return len(self.source_list)


def source_term(src, mesh):
    """Nodal right-hand side of one source (SimPEG or our own class)."""
    if hasattr(src, "eval_nodal"):
        return src.eval_nodal(mesh)
    locs = [np.asarray(src.location_a, float)]
    lb = getattr(src, "location_b", None)
    has_b = lb is not None and np.all(np.isfinite(np.asarray(lb, float)))
    if has_b:
        locs.append(np.asarray(lb, float))
    P = mesh.get_interpolation_matrix(np.vstack(locs), "N").toarray()
    cur = float(getattr(src, "current", 1.0))
    return cur * (P[0] - P[1]) if has_b else cur * P[0]
