"""Small OBJ/MTL scenes written by the tests themselves (no reference assets)."""
import os

BOX_MTL = """# materials of a closed box with an emitter
newmtl white
  Kd 0.73 0.73 0.73   # diffuse white
  Ke 0 0 0
  Ns 10
newmtl red
  Kd 0.63 0.06 0.05
newmtl green
  Kd 0.14 0.45 0.09
newmtl lamp
  Kd 0.78 0.78 0.78
  Ke 17 12 4
"""


def box_obj(nx=6, ny=6):
    """A 2x2x2 box open at z = -1 (facing the camera), walls as nx x ny quad grids
    addressed with negative indices, a 0.5 x 0.5 lamp quad just below the ceiling,
    and a tall block with per-vertex normals and uvs on its faces."""
    out = ["# test box", "mtllib box.mtl"]

    def grid(mtl, origin, du, dv):
        out.append(f"usemtl {mtl}")
        for i in range(nx):
            for j in range(ny):
                corners = []
                for (a, b) in ((i, j), (i + 1, j), (i + 1, j + 1), (i, j + 1)):
                    p = [origin[k] + du[k] * a / nx + dv[k] * b / ny for k in range(3)]
                    corners.append(p)
                for p in corners:
                    out.append("v %.6f %.6f %.6f" % tuple(p))
                out.append("f -4 -3 -2 -1")

    grid("white", (-1, -1, -1), (2, 0, 0), (0, 0, 2))     # floor
    grid("white", (-1, 1, -1), (0, 0, 2), (2, 0, 0))      # ceiling
    grid("white", (-1, -1, 1), (2, 0, 0), (0, 2, 0))      # back
    grid("red", (-1, -1, -1), (0, 2, 0), (0, 0, 2))       # left
    grid("green", (1, -1, -1), (0, 0, 2), (0, 2, 0))      # right
    out.append("usemtl lamp")
    for p in ((-0.25, 0.99, -0.25), (0.25, 0.99, -0.25), (0.25, 0.99, 0.25), (-0.25, 0.99, 0.25)):
        out.append("v %.6f %.6f %.6f" % p)
    out.append("f -4 -1 -2 -3")
    # block with normals / uvs (v/vt/vn and v//vn forms)
    out.append("usemtl white")
    base = [(-0.6, -1.0, 0.1), (-0.1, -1.0, 0.1), (-0.1, -1.0, 0.6), (-0.6, -1.0, 0.6)]
    top = [(x, 0.2, z) for (x, _, z) in base]
    for p in base + top:
        out.append("v %.6f %.6f %.6f" % p)
    for uv in ((0, 0), (1, 0), (1, 1), (0, 1)):
        out.append("vt %.3f %.3f" % uv)
    for n in ((0, 0, -1), (1, 0, 0), (0, 0, 1), (-1, 0, 0), (0, 1, 0)):
        out.append("vn %.1f %.1f %.1f" % n)
    # vertices of the block are the last 8: -8..-1; uvs -4..-1; normals -5..-1
    sides = [(-8, -7, -3, -4, -5), (-7, -6, -2, -3, -4), (-6, -5, -1, -2, -3), (-5, -8, -4, -1, -2)]
    for a, b, c, d, n in sides:
        out.append(f"f {a}/-4/{n} {b}/-3/{n} {c}/-2/{n} {d}/-1/{n}")
    out.append("f -4//-1 -3//-1 -2//-1 -1//-1")
    return "\n".join(out) + "\n"


def write_box(dirpath):
    with open(os.path.join(dirpath, "box.mtl"), "w") as f:
        f.write(BOX_MTL)
    p = os.path.join(dirpath, "box.obj")
    with open(p, "w") as f:
        f.write(box_obj())
    return p
