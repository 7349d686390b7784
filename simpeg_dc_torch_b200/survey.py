"""DC surveys: current sources and potential receivers.

Mirrors the attributes of SimPEG's `resistivity.sources`, `.receivers` and
`.survey.Survey` that the engines read (`source_list`, `receiver_list`,
`location_a/b` (or `location`), `locations_m/n` (or `locations`), `current`,
`data_type`), so a SimPEG survey object can be used in place of these
classes: the engines build the source terms and receiver projections from
those attributes alone (`source_term`, `receiver_projection`).

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


def source_electrodes(src):
    """(A, B) current electrode locations of a source (SimPEG's or ours); B is
    None for a pole (absent, None or NaN, as SimPEG writes a pole's B)."""
    loc = getattr(src, "location_a", None)
    a = np.asarray(src.location if loc is None else loc, float)
    lb = getattr(src, "location_b", None)
    if lb is None:
        return a, None
    lb = np.asarray(lb, float)
    return a, (lb if np.all(np.isfinite(lb)) else None)


def source_term(src, mesh):
    """Nodal right-hand side of one source (SimPEG or our own class):
    I (P_A - P_B) through nodal interpolation, B absent for a pole
    (SimPEG's `BaseSrc.eval` in the nodal formulation)."""
    if hasattr(src, "eval_nodal"):
        return src.eval_nodal(mesh)
    a, b = source_electrodes(src)
    locs = [a] if b is None else [a, b]
    P = mesh.get_interpolation_matrix(np.vstack(locs), "N").toarray()
    cur = float(getattr(src, "current", 1.0))
    return cur * (P[0] - P[1]) if b is not None else cur * P[0]


def receiver_projection(rx, mesh):
    """P (nD_rx, nN) of one receiver: P_M - P_N for a dipole, P_M for a pole,
    from the public locations of a SimPEG receiver or one of ours (what
    SimPEG's `rx.getP(mesh, "N")` returns, dctorch/simulation2d.py:236-244)."""
    import scipy.sparse as sp
    lm = getattr(rx, "locations_m", None)
    locs = getattr(rx, "locations", None)
    if lm is None:
        lm = locs[0] if isinstance(locs, (list, tuple)) else locs
    ln = getattr(rx, "locations_n", None)
    if ln is None and isinstance(locs, (list, tuple)) and len(locs) == 2:
        ln = locs[1]
    P = mesh.get_interpolation_matrix(np.atleast_2d(np.asarray(lm, float)), "N")
    if ln is not None:
        ln = np.atleast_2d(np.asarray(ln, float))
        if np.all(np.isfinite(ln)):
            P = P - mesh.get_interpolation_matrix(ln, "N")
    return sp.csr_matrix(P)
