"""Writes scenes as Wavefront OBJ text in the mixed styles a parser must
handle: coordinates in several decimal precisions, exponent and hexadecimal
forms, signs, tabs and padding; vn / vt / s / unknown lines and comments;
faces in the three formats of import_export/obj_import.cpp:209-224 (and quads,
whose fourth vertex the reference ignores); objects with usemtl; a material
library; CRLF line ends.  Seeded."""
import numpy as np

MATERIAL_PROPS = ["shell.density", "shell.heat_capacity", "shell.thermal_conductivity", "shell.thickness",
                  "front.specular_reflectance", "front.diffuse_reflectance", "front.absorbance",
                  "front.transmittance", "front.emissivity", "rear.specular_reflectance", "rear.diffuse_reflectance",
                  "rear.absorbance", "rear.transmittance", "rear.emissivity"]


def _num(x, rng):
    k = rng.integers(0, 8)
    x = float(np.float32(x))
    if k == 0:
        return "%.9g" % x
    if k == 1:
        return "%.17g" % x
    if k == 2:
        return "%e" % x
    if k == 3:
        return "%.3f" % x            # lossy: the parser must round these
    if k == 4:
        return float.hex(x)          # hexadecimal floating point
    if k == 5:
        return ("+%.8g" % x) if x >= 0 else "%.8g" % x
    if k == 6:
        return "%.40e" % x           # many digits
    return "%.6g" % x


def mtl_text(names, rng):
    lines = []
    for name in names:
        lines.append("# material %s" % name)
        lines.append("newmtl %s" % name)
        props = list(MATERIAL_PROPS)
        rng.shuffle(props)
        for p in props:
            if rng.random() < 0.1:
                lines.append("# a comment inside the block")
            lines.append("%s%s%s" % (p, " " if rng.random() < 0.8 else "\t", _num(rng.random(), rng)))
        lines.append("")  # the reference consumes the line after the last property
    return "\n".join(lines) + "\n"


def obj_text(faces, meshes=None, material_names=None, mtllib=None, seed=0, crlf=False):
    """OBJ text of faces (n, 9); meshes: (first, count) pairs (contiguous,
    in order) each written as an object with `usemtl` of material_names[k %
    len]; mtllib: the library file name written at the top."""
    rng = np.random.default_rng(seed)
    out = ["# generated scene", "mtllib %s" % mtllib] if mtllib else ["# generated scene"]
    faces = np.asarray(faces, np.float32).reshape(-1, 9)
    n = len(faces)
    bounds = {}
    if meshes is not None:
        for k, (first, count) in enumerate(meshes):
            bounds[first] = k
    for f in range(n):
        if f in bounds:
            k = bounds[f]
            out.append("%s mesh_%d" % ("o" if rng.random() < 0.5 else "g", k))
            if material_names:
                out.append("usemtl %s" % material_names[k % len(material_names)])
        for v in range(3):
            xyz = faces[f, 3 * v:3 * v + 3]
            sep = [" ", " ", "\t", "  "]
            out.append("v%s%s%s%s%s%s" % (sep[rng.integers(0, 4)], _num(xyz[0], rng), sep[rng.integers(0, 4)],
                                        _num(xyz[1], rng), sep[rng.integers(0, 4)], _num(xyz[2], rng)))
        r = rng.random()
        if r < 0.05:
            out.append("vn 0 0 1")
        elif r < 0.1:
            out.append("vt 0.5 0.5")
        elif r < 0.12:
            out.append("s off")
        elif r < 0.14:
            out.append("l 1 2")          # unknown directive: skipped
        elif r < 0.16:
            out.append("")
        i = 3 * f + 1
        form = rng.integers(0, 4)
        if form == 0:
            out.append("f %d %d %d" % (i, i + 1, i + 2))
        elif form == 1:
            out.append("f %d//%d %d//%d %d//%d" % (i, 1, i + 1, 1, i + 2, 1))
        elif form == 2:
            out.append("f %d/%d/%d %d/%d/%d %d/%d/%d" % (i, 1, 1, i + 1, 1, 1, i + 2, 1, 1))
        else:
            out.append("f %d %d %d %d" % (i, i + 1, i + 2, i))   # a quad: the fourth index is ignored
    text = "\n".join(out) + "\n"
    if crlf:
        text = text.replace("\n", "\r\n")
    return text.encode()
