"""Result files and landmarks of the registration application, host side.

* ``write_vtk`` / ``read_vtk``: legacy VTK structured points, the format SKMReg writes its results
  and checkpoints in through ITK's VTK image IO (include/IOUtils.h:40-50, src/SKMReg.cxx:468-525:
  ``df-full-<level>.vtk``, ``cp_image-<level>.vtk``, ``cp_jacdet-<level>.vtk``, ``warped.vtk``).
  Binary data is big-endian, as the format prescribes; ASCII files are read too.
* ``read_landmarks``: the POINTS text format of ReadLandmarks (include/IOUtils.h:67-103).
* ``target_registration_error``: CalculateTRE (include/itkUtils.h:268-293).
* ``write_results``: the files SKMReg leaves in its temp directory, from ``register`` outputs.
"""
from __future__ import annotations

import os

import numpy as np

_VTK_TYPES = {"float": ">f4", "double": ">f8", "int": ">i4", "unsigned_int": ">u4", "short": ">i2",
              "unsigned_short": ">u2", "char": "i1", "unsigned_char": "u1", "long": ">i8", "unsigned_long": ">u8"}


def write_vtk(path, array, spacing=None, origin=None, components=None, dtype="float", binary=True):
    """Writes an image (Y, X) / (Z, Y, X), a vector field (..., D) or a matrix field (..., D, D)
    as legacy VTK structured points.  ``components`` = number of trailing component axes (0 scalar,
    1 vector, 2 matrix); by default a trailing axis of length 2 or 3 on a 3-/4-dimensional
    array marks a vector field.  Vector fields of 2-D images get a zero third component (VECTORS
    carry three)."""
    a = np.asarray(array)
    if components is None:
        components = 1 if (a.ndim in (3, 4) and a.shape[-1] in (2, 3) and a.ndim - 1 == a.shape[-1]) else 0
    grid = a.shape[:a.ndim - components]
    D = len(grid)
    if D not in (2, 3):
        raise ValueError("image must be 2-D or 3-D")
    size = list(reversed(grid)) + [1] * (3 - D)
    sp = list(spacing) if spacing is not None else [1.0] * D
    org = list(origin) if origin is not None else [0.0] * D
    sp = [float(v) for v in sp] + [1.0] * (3 - D)
    org = [float(v) for v in org] + [0.0] * (3 - D)
    n = int(np.prod(grid))
    if components == 0:
        head = "SCALARS scalars %s 1\nLOOKUP_TABLE default\n" % dtype
        data = a.reshape(n)
    elif components == 1:
        c = a.shape[-1]
        flat = a.reshape(n, c)
        if c < 3:
            flat = np.concatenate([flat, np.zeros((n, 3 - c), flat.dtype)], axis=1)
        head = "VECTORS vectors %s\n" % dtype if flat.shape[1] == 3 else \
            "SCALARS scalars %s %d\nLOOKUP_TABLE default\n" % (dtype, flat.shape[1])
        data = flat
    else:
        m = a.reshape(n, -1)
        head = "SCALARS scalars %s %d\nLOOKUP_TABLE default\n" % (dtype, m.shape[1])
        data = m
    hdr = ("# vtk DataFile Version 3.0\nVTK File Generated by Insight Segmentation and Registration Toolkit (ITK)\n"
           "%s\nDATASET STRUCTURED_POINTS\nDIMENSIONS %d %d %d\nSPACING %.16e %.16e %.16e\nORIGIN %.16e %.16e %.16e\n"
           "POINT_DATA %d\n" % ("BINARY" if binary else "ASCII", size[0], size[1], size[2], sp[0], sp[1], sp[2],
                                org[0], org[1], org[2], n)) + head
    with open(path, "wb") as f:
        f.write(hdr.encode("ascii"))
        if binary:
            f.write(np.ascontiguousarray(data, dtype=_VTK_TYPES[dtype]).tobytes())
            f.write(b"\n")
        else:
            np.savetxt(f, np.asarray(data, np.float64).reshape(n, -1), fmt="%.17g")


def read_vtk(path):
    """Reads legacy VTK structured points (SCALARS with 1..n components, VECTORS or TENSORS).
    Returns (array in (Z, Y, X[, C]) order -- (Y, X[, C]) when the z extent is 1 --, spacing,
    origin), spacing and origin x first, as many entries as the image has axes."""
    with open(path, "rb") as f:
        raw = f.read()
    pos = 0

    def next_line():
        nonlocal pos
        end = raw.index(b"\n", pos)
        line = raw[pos:end].decode("ascii", "replace").strip()
        pos = end + 1
        return line

    binary, size, spacing, origin, npts, ncomp, vtype = None, None, [1.0] * 3, [0.0] * 3, None, 1, "float"
    kind = None
    while kind is None:
        line = next_line()
        if not line or line.startswith("#"):
            continue
        key = line.split()[0].upper()
        tok = line.split()
        if key in ("BINARY", "ASCII"):
            binary = key == "BINARY"
        elif key == "DATASET":
            if tok[1].upper() != "STRUCTURED_POINTS":
                raise ValueError("only STRUCTURED_POINTS datasets are supported")
        elif key == "DIMENSIONS":
            size = [int(v) for v in tok[1:4]]
        elif key in ("SPACING", "ASPECT_RATIO"):
            spacing = [float(v) for v in tok[1:4]]
        elif key == "ORIGIN":
            origin = [float(v) for v in tok[1:4]]
        elif key == "POINT_DATA":
            npts = int(tok[1])
        elif key == "SCALARS":
            vtype = tok[2]
            ncomp = int(tok[3]) if len(tok) > 3 else 1
            kind = "scalars"
        elif key == "VECTORS":
            vtype, ncomp, kind = tok[2], 3, "vectors"
        elif key == "TENSORS":
            vtype, ncomp, kind = tok[2], 9, "tensors"
    if kind == "scalars":
        save = pos
        line = next_line()
        if not line.upper().startswith("LOOKUP_TABLE"):
            pos = save
    if size is None or npts is None or binary is None:
        raise ValueError("incomplete VTK header")
    count = npts * ncomp
    if binary:
        dt = np.dtype(_VTK_TYPES[vtype])
        data = np.frombuffer(raw, dtype=dt, count=count, offset=pos).astype(np.float64)
    else:
        data = np.array(raw[pos:].split()[:count], dtype=np.float64)
    D = 3 if size[2] > 1 else 2
    grid = tuple(reversed(size[:D]))
    if ncomp == 1:
        arr = data.reshape(grid)
    elif kind == "tensors":
        arr = data.reshape(grid + (3, 3))
    else:
        arr = data.reshape(grid + (ncomp,))
        if kind == "vectors" and D == 2 and np.all(arr[..., 2] == 0):
            arr = arr[..., :2]
    return np.ascontiguousarray(arr), tuple(spacing[:D]), tuple(origin[:D])


def read_landmarks(path, dimensions):
    """ReadLandmarks (include/IOUtils.h:67-103): '#' comment lines, a 'POINTS n' line, then
    three coordinates per point (the first `dimensions` are kept).  Returns (n, D)."""
    pts = []
    declared = None
    with open(path) as f:
        for line in f:
            if line.startswith("#"):
                continue
            if line.startswith("POINTS"):
                declared = int(line.split()[1])
                continue
            vals = line.split()
            for k in range(0, len(vals) - 2, 3):
                try:
                    p = [float(v) for v in vals[k:k + 3]]
                except ValueError:
                    break
                pts.append(p[:dimensions])
    out = np.asarray(pts, np.float64).reshape(-1, dimensions)
    if declared is not None and declared != len(out):
        import warnings
        warnings.warn("number of points read (%d) differs from the header (%d)" % (len(out), declared))
    return out


def _interpolate_vector(field, spacing, origin, p):
    """Linear interpolation of a (..., D) field at physical point p; None outside the buffer
    ([-0.5, size - 0.5) in continuous index, neighbour indices clamped)."""
    D = field.shape[-1]
    size = tuple(reversed(field.shape[:-1]))
    ci = [(p[d] - origin[d]) / spacing[d] for d in range(D)]
    if any(not (-0.5 <= ci[d] < size[d] - 0.5) for d in range(D)):
        return None
    acc = np.zeros(D)
    base = [int(np.floor(c)) for c in ci]
    frac = [ci[d] - base[d] for d in range(D)]
    for corner in range(1 << D):
        w = 1.0
        idx = []
        for d in range(D):
            bit = (corner >> d) & 1
            w *= frac[d] if bit else 1.0 - frac[d]
            idx.append(min(max(base[d] + bit, 0), size[d] - 1))
        acc += w * field[tuple(reversed(idx))]
    return acc


def target_registration_error(displacement, spacing, origin, fixed_landmarks, moving_landmarks):
    """CalculateTRE (include/itkUtils.h:268-293): mean |T(moving_i) - fixed_i| with
    T(p) = p + u(p) (DisplacementFieldTransform, linearly interpolated, zero outside the field);
    -1 when the lists are empty or differ in length."""
    fl = np.asarray(fixed_landmarks, np.float64)
    ml = np.asarray(moving_landmarks, np.float64)
    if len(fl) == 0 or len(fl) != len(ml):
        return -1.0
    u = np.asarray(displacement, np.float64)
    D = u.shape[-1]
    spacing = tuple(spacing) if spacing is not None else (1.0,) * D
    origin = tuple(origin) if origin is not None else (0.0,) * D
    tre = 0.0
    for f, m in zip(fl, ml):
        v = _interpolate_vector(u, spacing, origin, m)
        q = m + (v if v is not None else 0.0)
        tre += float(np.linalg.norm(q - f))
    return tre / len(fl)


def write_results(directory, reference, displacement, spacing=None, origin=None, level_fields=None):
    """The files SKMReg writes (src/SKMReg.cxx:468-525): df.vtk, warped.vtk (order 1 resampling of
    the reference with the final field) and df-full-<level>.vtk for every given level field."""
    from .register import warp_image
    os.makedirs(directory, exist_ok=True)
    write_vtk(os.path.join(directory, "df.vtk"), displacement, spacing, origin, components=1)
    warped = warp_image(reference, displacement, spacing, origin, order=1)
    write_vtk(os.path.join(directory, "warped.vtk"), warped, spacing, origin, components=0)
    for level, field in sorted((level_fields or {}).items()):
        write_vtk(os.path.join(directory, "df-full-%d.vtk" % level), field, spacing, origin, components=1)
