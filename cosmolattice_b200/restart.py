"""Checkpoint and restart of a lattice run (SimulationManager::saveSim / loadSim / backup,
simulationmanager.h:69-141).

The reference writes an HDF5 file.  No HDF5 library is available to this build, so the same
variables go, in the same order, into a plain binary file:

    magic      16 bytes  b"CLB200-RESTART\\0\\0"
    header     8 x int64 version (1), model kind (clb_model_desc.kind), N, field components,
                         momentum components, sites per array (N^3), number of sectors, flags
                         (bit 0: the GW arrays are present)
    sectors    for each sector in the reference's save order (scalar singlets, complex scalars,
               SU(2) doublets, U(1) fields, SU(2) fields): its field components, then its momentum
               components, each N^3 float64 values in the order of clb_get_state; with the GW flag,
               after the scalar singlets (simulationmanager.h:112-114), the five GW field
               components each followed by its momentum component, N^3 float64 values each
    scalars    7 x float64   aSI, aI, aIM, aDotSI, aDotI, aDotSIM, tSave
    parameters int64 length, then the UTF-8 "key = value" lines of the run's parameters

Values are FP64 whatever the lattice's storage (the FP32 form's get_state returns FP64 values).
load_sim restores the state and then initializes in restart mode (CLB_INIT_RESTART): the cached
volume averages are refreshed (Averages::setAllAverages after loadSim) with no aDot correction,
and a leapfrog starts unsynced, as the reference's evolver does when it is constructed after a
restart (leapfrog.h:30-36).
"""
from __future__ import annotations

import os
import struct
from typing import Dict, List, Tuple

import numpy as np

MAGIC = b"CLB200-RESTART\0\0"
VERSION = 1
SCALARS = ("aSI", "aI", "aIM", "aDotSI", "aDotI", "aDotSIM")


def sectors(model) -> List[Tuple[str, range, range]]:
    """(name, field components, momentum components) per sector in the reference's save order
    (simulationmanager.h:112-125)."""
    if getattr(model, "NSU2", 0):  # S; phi; Phi; A; SU(2) links (quaternions) and momenta
        return [("scalar_0", range(0, 1), range(0, 1)), ("cmplx_scalar_0", range(1, 3), range(1, 3)),
                ("SU2Doublet_0", range(3, 7), range(3, 7)), ("U1_0", range(7, 10), range(7, 10)),
                ("SU2_0", range(10, 22), range(10, 19))]
    if getattr(model, "NU1", 0):
        return [("cmplx_scalar_0", range(0, 2), range(0, 2)), ("U1_0", range(2, 5), range(2, 5))]
    return [(f"scalar_{i}", range(i, i + 1), range(i, i + 1)) for i in range(model.Ns)]


FLAG_GWS = 1


def _gw_slot(secs) -> int:
    """Index of the first sector after the scalar singlets: where the GW arrays go."""
    k = 0
    while k < len(secs) and secs[k][0].startswith("scalar_"):
        k += 1
    return k


def save_sim(path: str, lattice, model, t: float, params: Dict[str, object] = None) -> None:
    """saveSim: the lattice's state, its GWs if enabled, scale factor and time (and the run's
    parameters) to path."""
    f, p, sf = lattice.get_state()
    N = lattice.rp.N
    n3 = N ** 3
    F = f.reshape(-1, n3)
    P = p.reshape(-1, n3)
    secs = sectors(model)
    gws = getattr(lattice, "gws_on", False)
    if gws:
        gu, gp = (a.reshape(5, n3) for a in lattice.gws_get_state())
    tmp = path + ".part"
    with open(tmp, "wb") as fh:
        fh.write(MAGIC)
        fh.write(struct.pack("<8q", VERSION, int(model.kind), N, F.shape[0], P.shape[0], n3, len(secs),
                             FLAG_GWS if gws else 0))
        for k in range(len(secs) + 1):
            if gws and k == _gw_slot(secs):
                for c in range(5):
                    fh.write(np.ascontiguousarray(gu[c], dtype="<f8").tobytes())
                    fh.write(np.ascontiguousarray(gp[c], dtype="<f8").tobytes())
            if k == len(secs):
                break
            _, fc, pc = secs[k]
            for c in fc:
                fh.write(np.ascontiguousarray(F[c], dtype="<f8").tobytes())
            for c in pc:
                fh.write(np.ascontiguousarray(P[c], dtype="<f8").tobytes())
        fh.write(struct.pack("<7d", *[float(sf[k]) for k in SCALARS], float(t)))
        text = "".join(f"{k} = {v}\n" for k, v in (params or {}).items()).encode()
        fh.write(struct.pack("<q", len(text)))
        fh.write(text)
    os.replace(tmp, path)


def _open(path: str):
    """The open restart file positioned after its header, and the header as a dict."""
    fh = open(path, "rb")
    try:
        if fh.read(16) != MAGIC:
            raise ValueError(f"{path}: not a restart file")
        version, kind, N, nf, npm, n3, nsec, flags = struct.unpack("<8q", fh.read(64))
        if version != VERSION:
            raise ValueError(f"{path}: restart format version {version}, expected {VERSION}")
    except Exception:
        fh.close()
        raise
    return fh, {"kind": kind, "N": N, "n_fields": nf, "n_momenta": npm, "n3": n3, "n_sectors": nsec,
                "gws": bool(flags & FLAG_GWS)}


def load_sim(path: str, lattice, model):
    """loadSim: the state of path into lattice (same model and N), its GWs if the lattice has them
    enabled (loadSim reads them only then; a lattice with GWs needs a file with them), then the
    cached averages.  Returns (t, parameter text)."""
    fh, hdr = _open(path)
    with fh:
        N = lattice.rp.N
        F = np.empty((hdr["n_fields"], hdr["n3"]))
        P = np.empty((hdr["n_momenta"], hdr["n3"]))
        if hdr["kind"] != int(model.kind) or hdr["N"] != N:
            raise ValueError(f"{path}: saved model kind {hdr['kind']} at N = {hdr['N']}, this run is kind "
                             f"{int(model.kind)} at N = {N}")
        gws = getattr(lattice, "gws_on", False)
        if gws and not hdr["gws"]:
            raise ValueError(f"{path}: the run has GWs, the restart file has none")
        n3 = hdr["n3"]
        secs = sectors(model)
        gu = gp = None
        for k in range(len(secs) + 1):
            if hdr["gws"] and k == _gw_slot(secs):
                pair = np.frombuffer(fh.read(8 * 10 * n3), dtype="<f8").reshape(5, 2, n3)
                gu, gp = pair[:, 0].copy(), pair[:, 1].copy()
            if k == len(secs):
                break
            _, fc, pc = secs[k]
            for c in fc:
                F[c] = np.frombuffer(fh.read(8 * n3), dtype="<f8")
            for c in pc:
                P[c] = np.frombuffer(fh.read(8 * n3), dtype="<f8")
        vals = struct.unpack("<7d", fh.read(56))
        (ln,) = struct.unpack("<q", fh.read(8))
        text = fh.read(ln).decode()
    sf = dict(zip(SCALARS, vals[:6]))
    lattice.set_state(F, P, sf)
    if gws:
        lattice.gws_set_state(gu.ravel(), gp.ravel())
    lattice.initialize(restart=True)
    return vals[6], text


def backup(folder: str, lattice, model, t: float, params: Dict[str, object] = None) -> str:
    """backup (simulationmanager.h:143-149): the previous backup is kept as <name>_backup.clb~."""
    path = os.path.join(folder, f"{model.name}_backup.clb")
    if os.path.exists(path):
        os.replace(path, path + "~")
    save_sim(path, lattice, model, t, params)
    return path
