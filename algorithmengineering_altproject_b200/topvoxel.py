"""Writing TopVoxel design-domain files (format version 1.0, read by `Problem.from_topvoxel`).

The format is the MATLAB original's external-model input (TOP3D_XL.m:458-586): whitespace-separated
tokens with 1-based, column-major indices

    voxel  k = 1 + y + nely * (x + nelx * z)              x < nelx, y < nely, z < nelz
    node   m = 1 + y + (nely+1) * (x + (nelx+1) * z)      x <= nelx, ...

`write_topvoxel` takes 0-based (x, y, z) coordinates and writes numbers with 17 significant digits, so
the reader recovers every load exactly.  `cantilever_topvoxel` writes the reference's built-in
cantilever (full cuboid, x = 0 face fixed, tip-line load, fea.cpp:374-403) as such a file.
"""
import numpy as np


def voxel_index(x, y, z, nelx, nely):
    return 1 + np.asarray(y) + nely * (np.asarray(x) + nelx * np.asarray(z))


def node_index(x, y, z, nelx, nely):
    return 1 + np.asarray(y) + (nely + 1) * (np.asarray(x) + (nelx + 1) * np.asarray(z))


def write_topvoxel(path, nelx, nely, nelz, solid, passive=(), fixations=(), loads=(), extra_load_cases=()):
    """solid, passive: iterables of (x, y, z) voxels; fixations: (x, y, z, fx, fy, fz) with 0/1 flags;
    loads: (x, y, z, Fx, Fy, Fz); extra_load_cases: lists of load rows (files the design loop refuses)."""
    def rows_of_loads(rows):
        return ["%d %.17g %.17g %.17g" % (node_index(x, y, z, nelx, nely), fx, fy, fz) for x, y, z, fx, fy, fz in rows]

    solid = [int(voxel_index(x, y, z, nelx, nely)) for x, y, z in solid]
    passive = [int(voxel_index(x, y, z, nelx, nely)) for x, y, z in passive]
    out = ["# TopVoxel design domain", "Version: 1.0", "Resolution: %d %d %d" % (nelx, nely, nelz),
           "Density values: 0", "Solid voxels: %d" % len(solid)]
    out += [str(k) for k in solid]
    out += ["Passive elements: %d" % len(passive)] + [str(k) for k in passive]
    out += ["Fixations: %d" % len(fixations)]
    out += ["%d %d %d %d" % (node_index(x, y, z, nelx, nely), fx, fy, fz) for x, y, z, fx, fy, fz in fixations]
    loads = list(loads)
    out += ["Loads: %d" % len(loads)] + rows_of_loads(loads)
    out += ["Additional loads: %d" % len(extra_load_cases)]
    for i, case in enumerate(extra_load_cases):
        case = list(case)
        out += ["Loads: %d %d" % (len(case), i + 2)] + rows_of_loads(case)
    with open(path, "w") as f:
        f.write("\n".join(out) + "\n")


def cantilever_topvoxel(path, nely, nelx, nelz, padded_res):
    """The reference cantilever as a TopVoxel file.  padded_res = (nx, ny, nz) of the padded grid
    (`Problem.res`): the tip load is F_z = -1/count on the nodes x = nelx, z <= max(1, nz // 6) of all
    (nely+1) rows, with count taken over the padded grid's (ny+1) rows as the reference does
    (fea.cpp:388-403); the load on padding nodes is dropped there because those nodes are fixed."""
    nx, ny, nz = padded_res
    iz_max = max(1, nz // 6)
    count = (iz_max + 1) * (ny + 1)
    solid = [(x, y, z) for z in range(nelz) for x in range(nelx) for y in range(nely)]
    fix = [(0, y, z, 1, 1, 1) for z in range(nelz + 1) for y in range(nely + 1)]
    loads = [(nelx, y, z, 0.0, 0.0, -1.0 / count) for z in range(min(iz_max, nelz) + 1) for y in range(nely + 1)]
    write_topvoxel(path, nelx, nely, nelz, solid, fixations=fix, loads=loads)
