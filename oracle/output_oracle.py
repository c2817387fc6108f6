"""Test infrastructure: restatements of tetmag's run artefacts, used only by tests/ to check the
library's writers and readers.

* ``log_header`` / ``log_row``: the .log file (writeLogFileHeader, main/TheSimulation.cpp:85-93;
  TheSimulation::writeLogStream, :367-372).  iostream's ``std::fixed`` / ``std::scientific`` /
  ``std::defaultfloat`` with a precision format like printf's ``%.Nf`` / ``%.Ne`` / ``%.Ng``; an
  Eigen row vector prints every coefficient right-aligned to the widest one, one space apart
  (Eigen's default IOFormat, which writeLogStream uses through ``getMeanM().transpose()``).
* ``vtk_xml`` / ``vtk_legacy``: magnetisation files in the encodings VTK's writers produce, the
  input of VTKReader::readMag (io/VTKReader.cpp:158-181): VTK XML with ASCII, inline base64
  (header and data as two base64 runs), appended base64 or appended raw arrays, optionally
  zlib-compressed in blocks (header: block count, block size, last block size, compressed sizes),
  UInt32 or UInt64 headers; legacy ASCII .vtk in the older CELLS layout and the version 5 one
  (OFFSETS / CONNECTIVITY).
"""
from __future__ import annotations

import base64
import struct
import zlib

import numpy as np


def log_header(start_time: str, host: str, user: str) -> str:
    """writeLogFileHeader (main/TheSimulation.cpp:85-93)."""
    return ("# Log file for simulation started " + start_time
            + "# on host " + host + " by user " + user + "\n"
            + "# data in the columns is: \n#(1) time in ps, (2) total energy , "
              "(3) demagnetizing energy, (4) exchange energy\n#(5) uniaxial anisotropy energy, "
              "(6) Zeeman energy, (7) cubic anisotropy energy (8) surface anisotropy energy, "
              "\n#(9) bulk DMI energy (10) maximum torque, (11-13) Mx, My, Mz, (14-16) Hx, Hy, Hz. "
              "All energies in J/m3, all fields in T\n")


def _eigen_row(strs) -> str:
    w = max(len(s) for s in strs)
    return " ".join(s.rjust(w) for s in strs)


ENERGY_KEYS = ("total", "demag", "exchange", "uniaxial", "zeeman", "cubic", "surface", "dmi")


def log_row(t_ps, energies, torque, mean_m, mean_h_tesla) -> str:
    """writeLogStream (main/TheSimulation.cpp:367-372)."""
    e = [energies[k] for k in ENERGY_KEYS] if isinstance(energies, dict) else list(energies)
    return ("%.4f" % t_ps + "".join("\t%.4f" % x for x in e) + "\t%.3e" % torque + "\t"
            + _eigen_row(["%.10g" % x for x in mean_m]) + "\t" + _eigen_row(["%.6f" % x for x in mean_h_tesla])
            + "\n")


# --------------------------------------------------------------------------------------------
# VTK files
# --------------------------------------------------------------------------------------------
def _payload(raw: bytes, header: str, compress: bool, block: int) -> tuple[bytes, bytes]:
    """(header bytes, data bytes) of one binary array."""
    fmt = "<Q" if header == "UInt64" else "<I"
    if not compress:
        return struct.pack(fmt, len(raw)), raw
    blocks = [raw[i:i + block] for i in range(0, len(raw), block)] or [b""]
    comp = [zlib.compress(b) for b in blocks]
    last = len(blocks[-1]) if len(blocks[-1]) != block else 0
    hdr = struct.pack("<" + fmt[1] * (3 + len(comp)), len(comp), block, last, *[len(c) for c in comp])
    return hdr, b"".join(comp)


def vtk_xml(xyz, tets, m_soa, time_ps=None, mode="appended-base64", header="UInt64", compress=True,
            dtype="Float64", block=32768, joint_base64=False) -> bytes:
    """A VTK XML unstructured grid with point array "Magnetization" (and "Material", "Points", cells)
    in one of VTK's encodings.  mode: "ascii", "binary" (inline base64), "appended-base64",
    "appended-raw".  joint_base64 encodes an uncompressed array's header and data as one run."""
    n = xyz.shape[0]
    m = np.asarray(m_soa).reshape(3, n).T.copy()
    npt = {"Float64": np.float64, "Float32": np.float32}[dtype]
    arrays = [("PointData", dtype, "Magnetization", 3, m.astype(npt)),
              ("PointData", "Int32", "Material", 1, np.zeros(n, np.int32)),
              ("Points", "Float32", "Points", 3, xyz.astype(np.float32)),
              ("Cells", "Int64", "connectivity", 1, np.asarray(tets, np.int64).ravel()),
              ("Cells", "Int64", "offsets", 1, 4 * np.arange(1, len(tets) + 1, dtype=np.int64)),
              ("Cells", "UInt8", "types", 1, np.full(len(tets), 10, np.uint8))]
    appended = []
    app_len = 0

    def data_array(typ, name, nc, a):
        nonlocal app_len
        att = f'type="{typ}" Name="{name}"' + (f' NumberOfComponents="{nc}"' if nc > 1 else "")
        if mode == "ascii":
            return f'<DataArray {att} format="ascii">\n' + " ".join(repr(float(x)) if a.dtype.kind == "f"
                                                                    else str(int(x)) for x in a.ravel()) \
                + "\n</DataArray>\n"
        h, d = _payload(a.tobytes(), header, compress, block)
        if mode == "appended-raw":
            off = app_len
            appended.append(h + d)
            app_len += len(h) + len(d)
            return f'<DataArray {att} format="appended" offset="{off}"/>\n'
        if joint_base64 and not compress:
            txt = base64.b64encode(h + d)
        else:
            txt = base64.b64encode(h) + base64.b64encode(d)
        if mode == "binary":
            return f'<DataArray {att} format="binary">\n' + txt.decode() + "\n</DataArray>\n"
        off = app_len
        appended.append(txt)
        app_len += len(txt)
        return f'<DataArray {att} format="appended" offset="{off}"/>\n'

    comp = ' compressor="vtkZLibDataCompressor"' if compress and mode != "ascii" else ""
    hdr_att = f' header_type="{header}"' if header == "UInt64" else ""
    out = [f'<?xml version="1.0"?>\n<VTKFile type="UnstructuredGrid" version="1.0" '
           f'byte_order="LittleEndian"{hdr_att}{comp}>\n<UnstructuredGrid>\n']
    if time_ps is not None:
        out.append('<FieldData>\n' + data_array("Float64", "timeInPs", 1, np.array([time_ps])) + '</FieldData>\n')
    out.append(f'<Piece NumberOfPoints="{n}" NumberOfCells="{len(tets)}">\n<PointData Scalars="Material" '
               f'Vectors="Magnetization">\n')
    for sec in ("PointData", "Points", "Cells"):
        if sec != "PointData":
            out.append(f"<{sec}>\n")
        for s, typ, name, nc, a in arrays:
            if s == sec:
                out.append(data_array(typ, name, nc, a))
        out.append(f"</{sec}>\n")
    out.append("</Piece>\n</UnstructuredGrid>\n")
    body = "".join(out).encode()
    if mode.startswith("appended"):
        enc = "raw" if mode == "appended-raw" else "base64"
        body += f'<AppendedData encoding="{enc}">\n_'.encode() + b"".join(appended) + b"\n</AppendedData>\n"
    return body + b"</VTKFile>\n"


def vtk_legacy(xyz, tets, m_soa, time_ps=None, layout="v5") -> str:
    """Legacy ASCII .vtk with POINT_DATA (Material scalars, Magnetization vectors)."""
    n = xyz.shape[0]
    m = np.asarray(m_soa).reshape(3, n).T
    ver = "5.1" if layout == "v5" else "4.2"
    s = [f"# vtk DataFile Version {ver}\nvtk output\nASCII\nDATASET UNSTRUCTURED_GRID\n"]
    if time_ps is not None:
        s.append(f"FIELD FieldData 1\ntimeInPs 1 1 double\n{time_ps!r}\n")
    s.append(f"POINTS {n} float\n" + "\n".join(" ".join(repr(float(c)) for c in p) for p in xyz) + "\n")
    ne = len(tets)
    if layout == "v5":
        s.append(f"CELLS {ne + 1} {4 * ne}\nOFFSETS vtktypeint64\n" + " ".join(str(4 * k) for k in range(ne + 1))
                 + "\nCONNECTIVITY vtktypeint64\n" + " ".join(str(int(i)) for i in np.ravel(tets)) + "\n")
    else:
        s.append(f"CELLS {ne} {5 * ne}\n" + "\n".join("4 " + " ".join(str(int(i)) for i in t) for t in tets) + "\n")
    s.append(f"CELL_TYPES {ne}\n" + "\n".join("10" for _ in range(ne)) + "\n")
    s.append(f"POINT_DATA {n}\nSCALARS Material int 1\nLOOKUP_TABLE default\n" + " ".join("0" for _ in range(n))
             + "\nVECTORS Magnetization double\n" + "\n".join(" ".join(repr(float(c)) for c in r) for r in m) + "\n")
    return "".join(s)
