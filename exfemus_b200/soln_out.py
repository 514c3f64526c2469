"""Solution output: MGEquationsSystem::print_soln (src/MGEquationsSystem.C:606-721) and
print_case (src/MGEquationsSystem.C:814-935) over the C ABI, XDMF text over raw binary
datasets in place of HDF5 (not installed here).

print_soln(systems, t_step, time, ...) writes the top level of one or more systems on
one mesh; print_case(systems, t_step, ...) writes their initial state with the boundary
flags; write_xdmf(...) writes node fields given as host arrays; read_xdmf(path) loads
a written step back (coordinates, sub-cell connectivity, node fields) by following the
XDMF file's Seek offsets, for checks and for restarting from output.
"""
import ctypes as C
import os
import xml.etree.ElementTree as ET

import numpy as np

from . import _lib
from ._lib import ExfNodeFields, ExfSolnOut, check


def _out(t_step, time, out_dir, basesol, basemesh, connlin, ndigits):
    o = ExfSolnOut()
    o.dir = (out_dir or "").encode()
    o.basesol = basesol.encode()
    o.basemesh = basemesh.encode()
    o.connlin = connlin.encode()
    o.ndigits = ndigits
    o.t_step = t_step
    o.time = time
    return o


def xmf_path(t_step, out_dir="", basesol="sol", ndigits=4):
    """Path of the XDMF file that print_soln / write_xdmf write for t_step."""
    return os.path.join(out_dir or "", "%s.%0*d.xmf" % (basesol, ndigits, t_step))


def print_soln(systems, t_step, time, out_dir="", basesol="sol", basemesh="mesh", connlin="_conn_lin",
               ndigits=4, names=None, refvalue=None):
    """Every variable of every system (MGSolNS: u, v[, w], p; MGSolT: T) at the top level,
    scaled by refvalue (one factor per variable, default 1), as XDMF time step t_step
    with <Time Value=time>.  Returns the XDMF file's path."""
    L = _lib.load()
    n = len(systems)
    hs = (C.c_void_p * n)(*[s.h for s in systems])
    nm = None
    if names is not None:
        nm = (C.c_char_p * len(names))(*[x.encode() for x in names])
    rv = None
    if refvalue is not None:
        rv = np.ascontiguousarray(refvalue, dtype=np.float64)
    o = _out(t_step, time, out_dir, basesol, basemesh, connlin, ndigits)
    check(L.exf_print_soln(hs, n, nm, None if rv is None else _lib.dptr(rv), C.byref(o)))
    return xmf_path(t_step, out_dir, basesol, ndigits)


def print_case(systems, t_step=0, out_dir="", basecase="case", basemesh="mesh", connlin="_conn_lin",
               ndigits=4, names=None, refvalue=None):
    """The initial state (x_old) of every variable of every system with its boundary
    flags, three node fields per variable: <name> (scaled by refvalue), <name>bd (bc[1],
    the Dirichlet flag) and <name>vl (bc[0], the value flag); the coordinates are those
    of <basemesh>.bin and the file has no <Time>.  Returns the XDMF file's path."""
    L = _lib.load()
    n = len(systems)
    hs = (C.c_void_p * n)(*[s.h for s in systems])
    nm = None
    if names is not None:
        nm = (C.c_char_p * len(names))(*[x.encode() for x in names])
    rv = None
    if refvalue is not None:
        rv = np.ascontiguousarray(refvalue, dtype=np.float64)
    o = _out(t_step, 0.0, out_dir, basecase, basemesh, connlin, ndigits)
    check(L.exf_print_case(hs, n, nm, None if rv is None else _lib.dptr(rv), C.byref(o)))
    return xmf_path(t_step, out_dir, basecase, ndigits)


def write_xdmf(dim, xyz, conn, fields, t_step=0, time=0.0, out_dir="", basesol="sol", basemesh="mesh",
               connlin="_conn_lin", ndigits=4, case=False):
    """Node fields on a quad9 / hex27 mesh given as host arrays: xyz [dim][nnodes], conn
    [nel][9 | 27], fields a list of (name, order, values[nnodes]) with order 2 for a
    quadratic variable and 1 for a linear one (read at the element vertices).  case=True
    writes a case file (the coordinates as <basemesh>.bin, no <Time>).  Returns the XDMF
    file's path."""
    L = _lib.load()
    xyz = np.ascontiguousarray(xyz, dtype=np.float64)
    conn = np.ascontiguousarray(conn, dtype=np.int32)
    nn = xyz.shape[1]
    vals = np.ascontiguousarray(np.array([f[2] for f in fields], dtype=np.float64).reshape(len(fields), nn))
    order = np.ascontiguousarray([f[1] for f in fields], dtype=np.int32)
    names = (C.c_char_p * max(1, len(fields)))(*[f[0].encode() for f in fields])
    nf = ExfNodeFields()
    nf.dim, nf.nnodes, nf.nel, nf.nvars = dim, nn, conn.shape[0], len(fields)
    nf.xyz, nf.conn = xyz.ctypes.data, conn.ctypes.data
    nf.names = names
    nf.order, nf.vals = order.ctypes.data, vals.ctypes.data
    o = _out(t_step, time, out_dir, basesol, basemesh, connlin, ndigits)
    check((L.exf_write_xdmf_case if case else L.exf_write_xdmf)(C.byref(nf), C.byref(o)))
    return xmf_path(t_step, out_dir, basesol, ndigits)


def _item(el, base):
    """The array a Binary DataItem / DataStructure addresses."""
    dims = [int(x) for x in el.get("Dimensions").split()]
    dt = {("Int", "4"): "<i4", ("Float", "8"): "<f8"}[(el.get("DataType"), el.get("Precision"))]
    if el.get("Endian") == "Big":
        dt = ">" + dt[1:]
    path = os.path.join(base, el.text.strip())
    count = int(np.prod(dims))
    a = np.fromfile(path, dtype=dt, count=count, offset=int(el.get("Seek", "0")))
    if a.size != count:
        raise ValueError("%s: short dataset" % path)
    return a.reshape(dims)


def read_xdmf(path):
    """A written step: {"time" (None for a case file), "cell_type", "cells" [nsub][4 | 8],
    "xyz" [3][nnodes], "fields" {name: [nnodes]}}."""
    base = os.path.dirname(path)
    grid = ET.parse(path).getroot().find("Domain").find("Grid")
    topo = grid.find("Topology")
    geo = grid.find("Geometry")
    out = {
        "time": None if grid.find("Time") is None else float(grid.find("Time").get("Value")),
        "cell_type": topo.get("Type"),
        "cells": _item(topo.find("DataStructure"), base),
        "xyz": np.stack([_item(d, base)[:, 0] for d in geo.findall("DataStructure")]),
        "fields": {},
    }
    for a in grid.findall("Attribute"):
        out["fields"][a.get("Name")] = _item(a.find("DataItem"), base)[:, 0]
    return out
