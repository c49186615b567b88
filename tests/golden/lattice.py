"""Regenerate the perfect-lattice model files the reference examples read.

The reference's examples/MorseTest/model.dump is an FCC lattice written by
LAMMPS (lattice fcc 3.68, region 0..10 in each direction, scaled coordinates
xs in multiples of 0.05).  Atom id 1+4n+b sits in unit cell
n = ix + 10*iy + 100*iz with basis b of (0,0,0), (.5,.5,0), (.5,0,.5),
(0,.5,.5).  The testCAF lattice (examples/testCAF/in.mX) is an 18^3
tessellation of a 3.629 A FCC cell from -9 to 9, written as xyz in Angstrom.
"""

BASIS = ((0.0, 0.0, 0.0), (0.5, 0.5, 0.0), (0.5, 0.0, 0.5), (0.0, 0.5, 0.5))


def _fmt(x):
    s = ("%.6f" % x).rstrip("0").rstrip(".")
    return s if s else "0"


def write_fcc_dump(path, cells, box):
    n = 4 * cells ** 3
    with open(path, "w") as f:
        f.write("ITEM: TIMESTEP\n0\nITEM: NUMBER OF ATOMS\n%d\n" % n)
        f.write("ITEM: BOX BOUNDS pp pp pp\n")
        for _ in range(3):
            f.write("0 %s\n" % _fmt(box))
        f.write("ITEM: ATOMS id type xs ys zs\n")
        for iz in range(cells):
            for iy in range(cells):
                for ix in range(cells):
                    cell = ix + cells * iy + cells * cells * iz
                    for b, (bx, by, bz) in enumerate(BASIS):
                        f.write("%d 1 %s %s %s\n" % (
                            1 + 4 * cell + b, _fmt((ix + bx) / cells),
                            _fmt((iy + by) / cells), _fmt((iz + bz) / cells)))


def _f32(x):
    import struct
    return struct.unpack("f", struct.pack("f", x))[0]


def write_fcc_xyz(path, cells, a, lo, tname):
    """Coordinates are single-precision products (cell index + basis) * a:
    with them the oracle reproduces the reference log's step-1 kinetic
    energy (0.163470E-16, which comes only from these rounding errors) to
    three digits, so the file the reference read was written that way."""
    n = 4 * cells ** 3
    af = _f32(a)
    with open(path, "w") as f:
        f.write("%d\n\n" % n)
        for iz in range(lo, lo + cells):
            for iy in range(lo, lo + cells):
                for ix in range(lo, lo + cells):
                    for bx, by, bz in BASIS:
                        f.write("%s %.9g %.9g %.9g\n" % (
                            tname, _f32(_f32(ix + bx) * af), _f32(_f32(iy + by) * af),
                            _f32(_f32(iz + bz) * af)))


def materialise(model, workdir):
    """Write the model file a golden script expects, relative to workdir."""
    import os
    path = os.path.normpath(os.path.join(workdir, model["file"]))
    os.makedirs(os.path.dirname(path), exist_ok=True)
    if model["kind"] == "fcc_dump":
        write_fcc_dump(path, model["cells"], model["box"])
    else:
        write_fcc_xyz(path, model["cells"], model["a"], model["lo"], model["type"])
    return path
