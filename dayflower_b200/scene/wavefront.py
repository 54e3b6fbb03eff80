"""Wavefront OBJ input: ``TriangleMesh3F.readWavefrontObject``
(``geometry/shape/TriangleMesh3F.java:534-740`` with its ``DefaultObjectModel``
and ``IndexedObjectModel``, ``:1200-1700``), producing :class:`TriangleMesh`
shapes the scene compiler takes.

Semantics kept from the reference:

* ``v``, ``vt``, ``vn``, ``f``, ``g``, ``o`` and ``usemtl`` statements; every
  other statement (and ``#`` comments) is skipped.
* A face of k vertices becomes k - 2 triangles fanned around its first vertex.
* Vertex references are 1-based ``v``, ``v/vt``, ``v//vn`` or ``v/vt/vn``; a
  missing texture coordinate is (0, 0).
* ``flip_texture_v`` stores 1 - v for every ``vt``.
* A file without any ``vn`` gets smooth normals: per position, the sum of the
  normalised face normals (edge AB x edge AC) of the triangles using it,
  normalised.
* ``scale`` multiplies positions and divides normals (the transpose of the
  inverse of a uniform scale), as ``Point4F.transformAndDivide`` and
  ``Vector3F.transformTranspose`` do.
* A new mesh starts wherever the group or the material name changes; each
  mesh keeps the group, material and object names current at its last
  triangle.

Where the reference's behaviour depends on malformed input (a file where only
some face vertices carry a normal misaligns its normal list), this reader uses
the face's geometric normal for the vertices without one.
"""
from __future__ import annotations

import io
import os
from typing import List, Union

import numpy as np

from .model import TriangleMesh


class WavefrontMesh(TriangleMesh):
    """A :class:`TriangleMesh` with the names ``readWavefrontObject`` gives its meshes."""

    def __init__(self, triangles, group_name: str, material_name: str, object_name: str):
        super().__init__(triangles)
        self.group_name, self.material_name, self.object_name = group_name, material_name, object_name


def _parse_ref(token: str, nv: int, nt: int, nn: int):
    parts = token.split("/")

    def idx(k, n):
        if len(parts) > k and parts[k] != "":
            i = int(parts[k]) - 1
            if not 0 <= i < n:
                raise ValueError("vertex reference %r out of range" % token)
            return i
        return -1

    return idx(0, nv), idx(1, nt), idx(2, nn)


def read_wavefront_obj(source: Union[str, os.PathLike, io.TextIOBase], flip_texture_v: bool = False,
                       scale: float = 1.0) -> List[WavefrontMesh]:
    """Reads an OBJ file (a path or an open text stream) into triangle meshes."""
    if isinstance(source, (str, os.PathLike)):
        with open(source, "r") as f:
            return read_wavefront_obj(f, flip_texture_v, scale)
    positions, uvs, normals = [], [], []
    corners = []  # per triangle corner: (position, uv, normal) indices, group, material, object
    group = material = obj = ""
    for line in source:
        el = line.split()
        if not el or el[0].startswith("#"):
            continue
        op = el[0]
        if op == "v":
            positions.append((float(el[1]), float(el[2]), float(el[3])))
        elif op == "vt":
            v = float(el[2]) if len(el) > 2 else 0.0
            uvs.append((float(el[1]), 1.0 - v if flip_texture_v else v))
        elif op == "vn":
            normals.append((float(el[1]), float(el[2]), float(el[3])))
        elif op == "g":
            group = el[1] if len(el) > 1 else ""
        elif op == "o":
            obj = el[1] if len(el) > 1 else ""
        elif op == "usemtl":
            material = el[1] if len(el) > 1 else ""
        elif op == "f":
            refs = [_parse_ref(t, len(positions), len(uvs), len(normals)) for t in el[1:]]
            for i in range(len(refs) - 2):
                corners.append((refs[0], refs[1 + i], refs[2 + i], group, material, obj))
    if not corners:
        return []
    P = np.asarray(positions, dtype=np.float32).reshape(-1, 3)
    T = np.asarray(uvs, dtype=np.float32).reshape(-1, 2)
    N = np.asarray(normals, dtype=np.float32).reshape(-1, 3)
    tri = np.array([[c[0][0], c[1][0], c[2][0]] for c in corners], dtype=np.int64)
    tex = np.array([[c[0][1], c[1][1], c[2][1]] for c in corners], dtype=np.int64)
    nor = np.array([[c[0][2], c[1][2], c[2][2]] for c in corners], dtype=np.int64)
    a, b, cc = P[tri[:, 0]], P[tri[:, 1]], P[tri[:, 2]]
    face = np.cross(b - a, cc - a)
    with np.errstate(invalid="ignore", divide="ignore"):
        face = face / np.linalg.norm(face, axis=1, keepdims=True)
    if N.shape[0] == 0:  # IndexedObjectModel.calculateNormals: smooth normals per position
        acc = np.zeros_like(P)
        for k in range(3):
            np.add.at(acc, tri[:, k], face)
        with np.errstate(invalid="ignore", divide="ignore"):
            smooth = acc / np.linalg.norm(acc, axis=1, keepdims=True)
        vn = [smooth[tri[:, k]] for k in range(3)]
    else:
        vn = [np.where((nor[:, k] >= 0)[:, None], N[np.maximum(nor[:, k], 0)], face) for k in range(3)]
    vt = [np.where((tex[:, k] >= 0)[:, None], T[np.maximum(tex[:, k], 0)] if T.shape[0] else 0.0, 0.0) for k in range(3)]
    rows = np.zeros((tri.shape[0], 24), dtype=np.float32)
    s = np.float32(scale)
    rows[:, 0:3], rows[:, 3:6], rows[:, 6:9] = a * s, b * s, cc * s
    rows[:, 9:11], rows[:, 11:13], rows[:, 13:15] = vt
    rows[:, 15:18], rows[:, 18:21], rows[:, 21:24] = vn[0] / s, vn[1] / s, vn[2] / s
    meshes: List[WavefrontMesh] = []
    start = 0
    for i in range(1, len(corners) + 1):
        if i == len(corners) or corners[i][3] != corners[i - 1][3] or corners[i][4] != corners[i - 1][4]:
            last = corners[i - 1]
            meshes.append(WavefrontMesh(rows[start:i], last[3], last[4], last[5]))
            start = i
    return meshes
