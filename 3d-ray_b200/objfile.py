"""Wavefront OBJ ingestion: the reference's direct path (no subdivision, no
displacement) from an OBJ file to the triangles of one mesh entity.

Restates `ObjLoader.Load` / `BuildTrianglesDirect`
(src/RayTracer/Scene/ObjLoader.cs:99-245, 357-400, 430-504):

- `v`, `vn` and `vt` lines are parsed in file order.
- Each `f` vertex is `v`, `v/vt`, `v/vt/vn` or `v//vn`. Indices are 1-based;
  negative ones count back from the entries read so far. An index that cannot
  be resolved leaves its channel missing for that vertex.
- A face has normals (UVs) only when every one of its vertices does. A channel
  that some faces have and others lack is dropped for the whole mesh.
- Faces are fan-triangulated around their first vertex. A triangle whose edge
  cross product has squared length under 1e-12 is skipped.
- Faces with normals become smooth triangles; the others stay flat.

Numbers are rounded once, straight to float32, as .NET's float.Parse does:
a float64 parse is used unless it lands exactly halfway between two float32
values, where the exact decimal decides.
"""
from __future__ import annotations

import dataclasses
from fractions import Fraction

import numpy as np


@dataclasses.dataclass
class ObjMesh:
    tris: np.ndarray               # [n, 9] float32: v0, v1, v2
    normals: np.ndarray | None     # [n, 9] float32: n0, n1, n2 (zeros for a flat face), or None
    uvs: np.ndarray | None         # [n, 6] float32: uv0, uv1, uv2, or None
    warnings: list


def _f32(tokens: list[str]) -> np.ndarray:
    """Correctly rounded float32 values of decimal strings."""
    d = np.array([float(t) for t in tokens], np.float64)
    f = d.astype(np.float32)
    # a float64 exactly halfway between two float32 neighbours may hide a
    # decimal on either side of the midpoint: decide those from the exact value
    up = np.nextafter(f, np.float32(np.inf)).astype(np.float64)
    dn = np.nextafter(f, np.float32(-np.inf)).astype(np.float64)
    fd = f.astype(np.float64)
    tie = np.isfinite(d) & ((d == (fd + up) / 2) | (d == (fd + dn) / 2))
    for i in np.nonzero(tie)[0]:
        exact = Fraction(tokens[i].strip())
        cands = [np.float32(fd[i]), np.float32(up[i]), np.float32(dn[i])]
        best = min(cands, key=lambda c: (abs(Fraction(float(c)) - exact),
                                         int(np.frombuffer(np.float32(c).tobytes(), np.uint32)[0]) & 1))
        f[i] = best
    return f


def _parse_index(s: str, size: int) -> int:
    """ObjLoader.TryParseIndex (:458-472): 1-based or negative, else -1."""
    try:
        raw = int(s.strip())
    except ValueError:
        return -1
    if raw > 0:
        idx = raw - 1
    elif raw < 0:
        idx = size + raw
    else:
        return -1
    return idx if 0 <= idx < size else -1


def load_obj(path: str) -> ObjMesh:
    """Parses `path` into the triangles ObjLoader.BuildTrianglesDirect builds."""
    warnings: list[str] = []
    pos_tok: list[str] = []
    nrm_tok: list[str] = []
    uv_tok: list[str] = []
    npos = nnrm = nuv = 0
    faces: list[tuple[list[int], list[int], list[int]]] = []
    with open(path, "r", encoding="utf-8", errors="replace") as fh:
        for line_num, raw in enumerate(fh, 1):
            line = raw.strip()
            if not line or line[0] == "#":
                continue
            if line.startswith("v "):
                parts = [t for t in line[2:].strip().split(" ") if t]
                if len(parts) >= 3 and all(_is_float(p) for p in parts[:3]):
                    pos_tok += parts[:3]
                    npos += 1
                else:
                    warnings.append(f"OBJ line {line_num}: malformed vertex position")
            elif line.startswith("vn "):
                parts = [t for t in line[3:].strip().split(" ") if t]
                if len(parts) >= 3 and all(_is_float(p) for p in parts[:3]):
                    nrm_tok += parts[:3]
                    nnrm += 1
                else:
                    warnings.append(f"OBJ line {line_num}: malformed vertex normal")
            elif line.startswith("vt "):
                parts = [t for t in line[3:].strip().split(" ") if t]
                if len(parts) >= 2 and all(_is_float(p) for p in parts[:2]):
                    uv_tok += parts[:2]
                    nuv += 1
                else:
                    warnings.append(f"OBJ line {line_num}: malformed texture coordinate")
            elif line.startswith("f "):
                fp, fn, fu = [], [], []
                for token in line[2:].split(" "):
                    if not token:
                        continue
                    sub = token.split("/", 2)
                    v = _parse_index(sub[0], npos)
                    if v < 0:
                        warnings.append(f"OBJ line {line_num}: malformed face vertex '{token}'")
                        continue
                    vt = _parse_index(sub[1], nuv) if len(sub) >= 2 and sub[1] else -1
                    vn = _parse_index(sub[2], nnrm) if len(sub) >= 3 and sub[2] else -1
                    fp.append(v)
                    fu.append(vt)
                    fn.append(vn)
                if len(fp) < 3:
                    warnings.append(f"OBJ line {line_num}: face has fewer than 3 vertices, skipping")
                    continue
                faces.append((fp, fn if min(fn) >= 0 else [], fu if min(fu) >= 0 else []))
    if not faces:
        raise ValueError(f"{path}: OBJ file produced zero faces")
    pos = _f32(pos_tok).reshape(-1, 3)
    nrm = _f32(nrm_tok).reshape(-1, 3) if nnrm else np.zeros((0, 3), np.float32)
    uvs = _f32(uv_tok).reshape(-1, 2) if nuv else np.zeros((0, 2), np.float32)
    has_n = [bool(f[1]) for f in faces]
    has_u = [bool(f[2]) for f in faces]
    use_n = any(has_n) and all(has_n)    # a partial channel is dropped (ObjLoader.cs:205-208)
    use_u = any(has_u) and all(has_u)
    tris, tn, tu = [], [], []
    for fp, fn, fu in faces:
        for k in range(1, len(fp) - 1):
            v0, v1, v2 = pos[fp[0]], pos[fp[k]], pos[fp[k + 1]]
            e1 = (v1 - v0).astype(np.float32)
            e2 = (v2 - v0).astype(np.float32)
            cr = np.array([e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2],
                           e1[0] * e2[1] - e1[1] * e2[0]], np.float32)
            if np.float32(np.float32(cr[0] * cr[0] + cr[1] * cr[1]) + cr[2] * cr[2]) < np.float32(1e-12):
                continue
            tris.append(np.concatenate([v0, v1, v2]))
            if use_n:
                tn.append(np.concatenate([nrm[fn[0]], nrm[fn[k]], nrm[fn[k + 1]]]))
                if use_u:
                    tu.append(np.concatenate([uvs[fu[0]], uvs[fu[k]], uvs[fu[k + 1]]]))
    if not tris:
        raise ValueError(f"{path}: OBJ file produced zero triangles")
    return ObjMesh(np.asarray(tris, np.float32).reshape(-1, 9),
                   np.asarray(tn, np.float32).reshape(-1, 9) if use_n else None,
                   np.asarray(tu, np.float32).reshape(-1, 6) if use_n and use_u else None,
                   warnings)


def _is_float(s: str) -> bool:
    try:
        float(s)
        return True
    except ValueError:
        return False


def write_obj(path: str, tris: np.ndarray, normals: np.ndarray | None = None, uvs: np.ndarray | None = None):
    """Writes triangles (and, for smooth ones, vertex normals and UVs) as an
    OBJ that `load_obj` and the reference's ObjLoader read back to the same
    float32 values (9 significant digits round-trip a float32)."""
    tris = np.asarray(tris, np.float32).reshape(-1, 3, 3)
    with open(path, "w") as fh:
        for t in tris:
            for v in t:
                fh.write("v {:.9g} {:.9g} {:.9g}\n".format(*map(float, v)))
        if normals is not None:
            for n in np.asarray(normals, np.float32).reshape(-1, 3):
                fh.write("vn {:.9g} {:.9g} {:.9g}\n".format(*map(float, n)))
        if uvs is not None:
            for uv in np.asarray(uvs, np.float32).reshape(-1, 2):
                fh.write("vt {:.9g} {:.9g}\n".format(*map(float, uv)))
        for i in range(tris.shape[0]):
            a, b, c = 3 * i + 1, 3 * i + 2, 3 * i + 3
            if normals is not None and uvs is not None:
                fh.write(f"f {a}/{a}/{a} {b}/{b}/{b} {c}/{c}/{c}\n")
            elif normals is not None:
                fh.write(f"f {a}//{a} {b}//{b} {c}//{c}\n")
            else:
                fh.write(f"f {a} {b} {c}\n")
