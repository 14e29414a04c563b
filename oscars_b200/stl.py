"""STL meshes for the power density on facets.

Restates the reference's containers: TTriangle3DContainer::ReadSTLFile / WriteSTLFile
(src/TTriangle3DContainer.cc:109-270), TSTLContainer (src/TSTLContainer.cc) and the facet values
of TTriangle3D (src/TTriangle3D.cc).

* Binary STL only: an 80-byte header, a uint32 triangle count, then per triangle the normal and the
  three vertices as float32 and a uint16 attribute.
* Vertices are the stored floats times ``scale`` (in double); normals are kept as stored (not
  normalised, not rotated).  Each facet's centre is ((A + B) + C) / 3 of the scaled vertices; the
  translation is then added to the vertices and to the centre.
* The reference resets the rotation angles to zero before it applies them, so ``rotations`` has no
  effect on the mesh (it is accepted and shown as (0, 0, 0) by print_stl, as there).
* Objects are named "_stl<k>" (k = objects held) unless a name is given; a repeated name is refused.
"""
from __future__ import annotations

import numpy as np

_RECORD = np.dtype([("n", "<f4", (3,)), ("a", "<f4", (3,)), ("b", "<f4", (3,)), ("c", "<f4", (3,)),
                    ("attr", "<u2")])
_HEADER = b"OSCARS OSCARS OSCARS OSCARS OSCARS   "


class StlMesh:
    """One imported STL object: facets (n x 12 = A, B, C, stored normal) and centres (n x 3)."""

    def __init__(self, name, filename, scale, translation, facets, centers):
        self.name = name
        self.filename = filename
        self.scale = scale
        self.translation = translation
        self.facets = facets
        self.centers = centers

    def __len__(self):
        return self.facets.shape[0]


def read_stl(path, scale=1.0, translation=(0.0, 0.0, 0.0), name=""):
    try:
        with open(path, "rb") as f:
            data = f.read()
    except OSError:
        raise ValueError("input file cannot be opened")
    if len(data) < 84:
        raise ValueError("input file is not a binary STL file")
    n = int(np.frombuffer(data, dtype="<u4", count=1, offset=80)[0])
    if len(data) < 84 + 50 * n:
        raise ValueError("input file is shorter than its triangle count")
    rec = np.frombuffer(data, dtype=_RECORD, count=n, offset=84)
    scale = float(scale)
    A = rec["a"].astype(np.float64) * scale
    B = rec["b"].astype(np.float64) * scale
    C = rec["c"].astype(np.float64) * scale
    centers = ((A + B) + C) / 3.0
    T = np.asarray(translation, dtype=np.float64).reshape(1, 3)
    facets = np.hstack([A + T, B + T, C + T, rec["n"].astype(np.float64)])
    return StlMesh(name, path, scale, [float(v) for v in T.ravel()], np.ascontiguousarray(facets),
                   np.ascontiguousarray(centers + T))


def _g(v):
    return "%g" % v


class StlContainer:
    """The STL objects of a simulation, facets in the order the objects were added."""

    def __init__(self):
        self.meshes: list[StlMesh] = []

    def add(self, path, scale=1.0, translation=(0.0, 0.0, 0.0), name=""):
        my_name = name if name else "_stl%d" % len(self.meshes)
        if any(m.name == my_name for m in self.meshes):
            raise ValueError("stl with this name already exists")
        self.meshes.append(read_stl(path, scale, translation, my_name))

    def remove(self, name):
        self.meshes = [m for m in self.meshes if m.name != name]

    def clear(self):
        self.meshes = []

    def __len__(self):
        return sum(len(m) for m in self.meshes)

    def facets(self):
        if not self.meshes:
            return np.zeros((0, 12)), np.zeros((0, 3))
        return (np.ascontiguousarray(np.vstack([m.facets for m in self.meshes])),
                np.ascontiguousarray(np.vstack([m.centers for m in self.meshes])))

    def write_stl(self, path):
        """TSTLContainer::WriteSTLFile: every facet of every object, vertices times the object's scale
        once more (as the reference writes them) and normals, as float32, attribute 0.  The 80-byte
        header holds the reference's text followed by zero bytes."""
        facets = np.vstack([np.hstack([m.facets[:, 0:9] * m.scale, m.facets[:, 9:12]]) for m in self.meshes]) \
            if self.meshes else np.zeros((0, 12))
        rec = np.zeros(facets.shape[0], dtype=_RECORD)
        rec["n"] = facets[:, 9:12]
        rec["a"] = facets[:, 0:3]
        rec["b"] = facets[:, 3:6]
        rec["c"] = facets[:, 6:9]
        try:
            with open(path, "wb") as f:
                f.write(_HEADER.ljust(80, b"\0"))
                f.write(np.array([facets.shape[0]], dtype="<u4").tobytes())
                f.write(rec.tobytes())
        except OSError:
            raise ValueError("output file cannot be opened")

    def describe(self):
        """The text of print_stl (the TSTLContainer and TTriangle3DContainer printers)."""
        out = "*STL Information*\nTSTLContainer has %d STL Objects\n" % len(self.meshes)
        for m in self.meshes:
            t = m.translation
            out += ("Name:             %s\nFilenName:        %s\nScale:            %s\nRotations:        (0, 0, 0)\n"
                    "Translation:      (%s, %s, %s)\nNTriangles:       %d\n\n"
                    % (m.name, m.filename, _g(m.scale), _g(t[0]), _g(t[1]), _g(t[2]), len(m)))
        return out + "\n"
