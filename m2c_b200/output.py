"""Solution snapshots in the reference's format: VTK rectilinear-grid files
(.vtr), one per frame, named <base>_<frame padded to 4 digits>.vtr, with the
reference's field names (Output::WriteSolutionSnapshot, Output.cpp:145-330):
density, velocity (3 components), pressure, materialid and levelset<k>,
given at the cell centres (the DMDA's coordinates).

The state comes from the device in one call (m2cg_download_state, the
ghosted host layout); the file is written on the host with its arrays
appended as raw little-endian binary.
"""
import struct

import numpy as np

from . import abi


def _coords(g):
    return abi.cell_centres(g)


def frame_name(base, frame):
    """Output.cpp:156-180: 4-digit zero padding up to 9999."""
    return f"{base}_{frame:04d}.vtr"


def write_vtr(path, g, V, ID=None, phi=None, fields=("density", "velocity", "pressure", "materialid", "levelset0")):
    """Write one snapshot. V, ID, phi: ghosted host arrays (as downloaded);
    only interior cells are written."""
    nx, ny, nz = g.nx, g.ny, g.nz
    inner = np.s_[1:-1, 1:-1, 1:-1]
    arrays = []
    Vi = np.asarray(V)[inner]
    for f in fields:
        if f == "density":
            arrays.append((f, 1, Vi[..., 0]))
        elif f == "velocity":
            arrays.append((f, 3, Vi[..., 1:4]))
        elif f == "pressure":
            arrays.append((f, 1, Vi[..., 4]))
        elif f == "materialid" and ID is not None:
            arrays.append((f, 1, np.asarray(ID)[inner]))
        elif f.startswith("levelset") and phi is not None:
            arrays.append((f, 1, np.asarray(phi)[inner]))
    xs = _coords(g)
    blobs, heads = [], []
    offset = 0

    def add(name, ncomp, data):
        nonlocal offset
        raw = np.ascontiguousarray(data, dtype="<f8").tobytes()
        heads.append((name, ncomp, offset))
        blobs.append(struct.pack("<Q", len(raw)) + raw)
        offset += 8 + len(raw)

    coord_heads = []
    for a, name in enumerate(("x", "y", "z")):
        coord_heads.append(offset)
        add(name, 1, xs[a])
    coord_heads_names = heads[:3]
    heads.clear()
    for name, ncomp, data in arrays:
        add(name, ncomp, data)
    ext = f"0 {nx - 1} 0 {ny - 1} 0 {nz - 1}"
    lines = ['<?xml version="1.0"?>',
             '<VTKFile type="RectilinearGrid" version="1.0" byte_order="LittleEndian" header_type="UInt64">',
             f'  <RectilinearGrid WholeExtent="{ext}">', f'    <Piece Extent="{ext}">', '      <Coordinates>']
    for (name, _, off) in coord_heads_names:
        lines.append(f'        <DataArray type="Float64" Name="{name}" NumberOfComponents="1" format="appended" '
                     f'offset="{off}"/>')
    lines += ['      </Coordinates>', '      <PointData>']
    for (name, ncomp, off) in heads:
        lines.append(f'        <DataArray type="Float64" Name="{name}" NumberOfComponents="{ncomp}" '
                     f'format="appended" offset="{off}"/>')
    lines += ['      </PointData>', '    </Piece>', '  </RectilinearGrid>', '  <AppendedData encoding="raw">']
    with open(path, "wb") as fh:
        fh.write(("\n".join(lines) + "\n   _").encode())
        for b in blobs:
            fh.write(b)
        fh.write(b"\n  </AppendedData>\n</VTKFile>\n")


def read_vtr(path):
    """Arrays of a file written by write_vtr: {name: array} (coordinates
    x, y, z and the point data, vectors as [n][3]), for checks."""
    raw = open(path, "rb").read()
    head, data = raw.split(b"   _", 1)
    out = {}
    import re
    for m in re.finditer(rb'Name="(\w+)" NumberOfComponents="(\d+)" format="appended" offset="(\d+)"', head):
        name, ncomp, off = m.group(1).decode(), int(m.group(2)), int(m.group(3))
        n = struct.unpack("<Q", data[off:off + 8])[0]
        arr = np.frombuffer(data[off + 8:off + 8 + n], dtype="<f8")
        out[name] = arr.reshape(-1, ncomp) if ncomp > 1 else arr
    return out


class Snapshots:
    """Frames of a solver every `every` steps: advance in chunks with the
    state resident on the device, download once per frame, write the file."""

    def __init__(self, solver, base, every):
        self.solver, self.base, self.every, self.frame = solver, base, every, 0

    def write(self):
        V, ID, phi = self.solver.download()
        path = frame_name(self.base, self.frame)
        write_vtr(path, self.solver.g, V, ID, phi)
        self.frame += 1
        return path

    def run(self, nsteps):
        done = 0
        paths = [self.write()]
        while done < nsteps:
            k = min(self.every, nsteps - done)
            self.solver.run(k)
            done += k
            paths.append(self.write())
        return paths
