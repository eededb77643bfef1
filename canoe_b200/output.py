"""NetCDF output of MeshBlock states in the reference's file layout, and the
regression check its example runs are judged by.

Layout (NetcdfOutput::WriteOutputFile, src/outputs/netcdf.cpp:45-470):

- one classic-format file per MeshBlock and output number,
  ``<basename>.block<gid>.<file_id>.<number:05d>.nc`` (netcdf.cpp:83-99);
  the per-block files of one output are combined into
  ``<basename>.<file_id>.<number:05d>.nc`` (NetcdfOutput::CombineBlocks,
  src/outputs/combine_blocks.cpp:19-60, which runs mppnccombine), the same
  file the pnetcdf writer makes in one go (src/outputs/pnetcdf.cpp:62-72);
- dimensions ``time`` (unlimited), ``x1``, ``x2``, ``x3`` and, where a
  direction has more than one cell, ``x1f`` / ``x2f`` / ``x3f``
  (netcdf.cpp:106-134);
- coordinate variables ``x1`` / ``x2`` / ``x3`` (axes Z / Y / X) and their
  faces, each carrying ``domain_decomposition`` = [first, last] of the whole
  mesh and [first, last] of this block, cells counted from 1 and faces from
  0 (netcdf.cpp:147-207);
- every cell variable NC_FLOAT on (time, x1, x2, x3), i.e. the transpose of
  the block's (k, j, i) layout (netcdf.cpp:446-454), with the units and long
  name of the metadata table (src/outputs/output_utils.cpp:31-47).

Variables: ``prim`` is the hydro primitive state, rho / press / vel1-3, plus
one mass fraction per species slot, named after the species
(src/outputs/load_user_output_data.cpp:27-36); ``uov`` holds the
temperature and the potential temperature T (p0 / p)^((gamma_d - 1) /
gamma_d), as the rising-bubble example computes them before every output
(examples/2019-Li-snap/robert.cpp:37-61), T = p / (rho R_d f_eps) the ideal
moist equation of state.

The regression check restates examples/2019-Li-snap/test_robert.py,
test_straka.py and test_bryan.py: the L2 norm, sqrt(sum(d^2)), of the
difference of one variable's slice between two output files, against the
threshold of each example.

    python -m canoe_b200.output robert new.nc golden.nc
"""
import glob
import os
import re
import sys

import numpy as np
from scipy.io import netcdf_file

from ._abi import NGHOST

# short name -> (long name, units): the entries of the metadata table
# (output_utils.cpp:31-47) this path writes
META = {
    "x1": ("height at cell center", "m"),
    "x1f": ("height at cell boundary", "m"),
    "x2": ("distance at cell center", "m"),
    "x2f": ("distance at cell boundary", "m"),
    "x3": ("distance at cell center", "m"),
    "x3f": ("distance at cell boundary", "m"),
    "rho": ("density", "kg/m^3"),
    "press": ("pressure", "pa"),
    "vel1": ("vertical velocity", "m/s"),
    "vel2": ("horizontal velocity", "m/s"),
    "vel3": ("horizontal velocity", "m/s"),
    "temp": ("temperature", "K"),
    "theta": ("potential temperature", "K"),
    "theta_e": ("equivalent potential temperature", "K"),
}

# (axis letter, long name of the centres, long name of the faces) of the
# coordinate variables (netcdf.cpp:147-207)
_AXES = {
    1: ("Z", "Z-coordinate at cell center", "Z-coordinate at cell face"),
    2: ("Y", "Y-coordinate at cell center", "Y-coordinate at cell face"),
    3: ("X", "X-coordinate at cell center", "X-coordinate at cell face"),
}

VAPOR_NAMES = ("H2O", "NH3", "H2S", "CH4")

# the regression checks of the examples: (variable, slice of the variable,
# threshold on the L2 norm of the difference)
CHECKS = {
    # test_robert.py: theta[-1, :, :, :] < 10
    "robert": ("theta", (-1, slice(None), slice(None), slice(None)), 10.0),
    # test_straka.py: theta[-1, :, :, 0] < 50
    "straka": ("theta", (-1, slice(None), slice(None), 0), 50.0),
    # test_bryan.py: theta_e[3, 0, :, :] < 900
    "bryan": ("theta_e", (3, 0, slice(None), slice(None)), 900.0),
}


def species_names(th, vapors=None):
    """Names of the mass-fraction slots 1..ny: the vapours, then their
    liquids "(l)", then their ices "(s)" (the slot order of the thermo
    parameter sets)."""
    nv = th.nvapor
    vapors = list(vapors or VAPOR_NAMES[:nv])
    names = list(vapors)
    if th.ny > nv:
        names += [f"{v}(l)" for v in vapors]
    if th.ny > 2 * nv:
        names += [f"{v}(s)" for v in vapors]
    if len(names) != th.ny:
        names = [f"q{n}" for n in range(1, th.ny + 1)]
    return names


def coordinates(cfg, x1f):
    """Cell centres and faces of a block: {"x1": ..., "x1f": ..., ...}."""
    x1f = np.asarray(x1f, dtype=np.float64)
    out = {"x1f": x1f, "x1": 0.5 * (x1f[1:] + x1f[:-1])}
    for d, (n, lo, dx) in {2: (cfg.nx2, cfg.x2min, cfg.dx2),
                           3: (cfg.nx3, cfg.x3min, cfg.dx3)}.items():
        f = lo + dx * np.arange(n + 1)
        out[f"x{d}f"] = f
        out[f"x{d}"] = 0.5 * (f[1:] + f[:-1])
    return out


def cell_fields(cfg, w, variables=("prim", "uov"), p0=1.0e5, species=None):
    """{name: (nx1, nx2, nx3) array} of a block's primitive state w
    (NV, nc3, nc2, nc1), interior cells only, in writing order."""
    th = cfg.thermo
    ny = th.ny
    ks = NGHOST if cfg.nx3 > 1 else 0
    js = NGHOST if cfg.nx2 > 1 else 0
    wi = w[:, ks:ks + cfg.nx3, js:js + cfg.nx2, NGHOST:NGHOST + cfg.nx1]
    wi = np.transpose(wi, (0, 3, 2, 1))  # (n, i, j, k)
    out = {}
    rho, q, pres = wi[0], wi[1:1 + ny], wi[4 + ny]
    if "prim" in variables:
        out["rho"] = rho
        out["press"] = pres
        for d in range(3):
            out[f"vel{d + 1}"] = wi[1 + ny + d]
        for name, qn in zip(species or species_names(th), q):
            out[name] = qn
    if "uov" in variables or "theta_e" in variables:
        feps = np.ones_like(rho)
        for n in range(ny):
            feps = feps + (q[n] * th.inv_mu_ratio_m1[n] if n < th.nvapor else -q[n])
        temp = pres / (rho * th.rd * feps)
        if "uov" in variables:
            chi = (th.gammad - 1.0) / th.gammad
            out["temp"] = temp
            out["theta"] = temp * (p0 / pres) ** chi
        if "theta_e" in variables:
            # the moist bubble's output (bryan.cpp:62-90)
            from . import thermo
            out["theta_e"] = thermo.theta_e(th, q, temp, pres, p0)
    return out


def write_file(path, coords, fields, time, decomposition=None, nfiles=1):
    """One classic NetCDF file with one time record.  decomposition:
    {d: (mesh_n, first)} per direction d = 1..3 (cells of the mesh, the
    block's first cell counted from 0) for the domain_decomposition
    attributes of a per-block file; None for a whole-domain file."""
    n = {d: len(coords[f"x{d}"]) for d in (1, 2, 3)}
    with netcdf_file(path, "w", version=1) as f:
        f.createDimension("time", None)
        for d in (1, 2, 3):
            f.createDimension(f"x{d}", n[d])
            if n[d] > 1:
                f.createDimension(f"x{d}f", n[d] + 1)
        v = f.createVariable("time", "f4", ("time",))
        v.axis, v.units, v.long_name = "T", "s", "time"
        v[0] = np.float32(time)
        for d in (1, 2, 3):
            axis, lc, lf = _AXES[d]
            v = f.createVariable(f"x{d}", "f4", (f"x{d}",))
            v.axis, v.units, v.long_name = axis, "m", lc
            v[:] = coords[f"x{d}"].astype(np.float32)
            if decomposition is not None:
                mesh_n, first = decomposition[d]
                v.domain_decomposition = np.array([1, mesh_n, first + 1, first + n[d]],
                                                  dtype=np.int32)
            if n[d] > 1:
                v = f.createVariable(f"x{d}f", "f4", (f"x{d}f",))
                v.units, v.long_name = "m", lf
                v[:] = coords[f"x{d}f"].astype(np.float32)
                if decomposition is not None:
                    mesh_n, first = decomposition[d]
                    v.domain_decomposition = np.array([0, mesh_n, first, first + n[d]],
                                                      dtype=np.int32)
        f.NumFilesInSet = np.int32(nfiles)
        for name, a in fields.items():
            v = f.createVariable(name, "f4", ("time", "x1", "x2", "x3"))
            if name in META:
                v.long_name, v.units = META[name]
            v[0] = a.astype(np.float32)


def block_filename(basename, gid, file_id, number):
    return f"{basename}.block{gid}.{file_id}.{number:05d}.nc"


def combined_filename(basename, file_id, number):
    return f"{basename}.{file_id}.{number:05d}.nc"


def _blocks_of(source):
    """[(cfg, x1f, w, (o1, o2, o3))] of a MeshBlock-like object (problem,
    primitive()) or a Mesh (split, blocks); offsets in cells of the mesh."""
    split = getattr(source, "split", None)
    if split is not None:
        if hasattr(source, "synchronize"):
            source.synchronize()
        return [(p.cfg, p.x1f, b.primitive(), (0, o2, o3))
                for p, b, (o2, o3) in zip(split.blocks, source.blocks, split.offsets)]
    p = source.problem
    return [(p.cfg, p.x1f, source.primitive(), (0, 0, 0))]


class NetcdfOutput:
    """One ``<output>`` block of file type netcdf: at every output the
    primitive state of each MeshBlock of the source goes to its own file,
    and (combine=True) the files are joined into the whole-domain file.
    Outputs are due at the start, whenever the time has reached next_time,
    and at the end (Outputs::MakeOutputs; main.cpp:94-95, 137-140); each
    output advances next_time by dt and the file number by one
    (netcdf.cpp:472-476)."""

    def __init__(self, basename, dt, file_id="out2", variables=("prim", "uov"), p0=1.0e5,
                 species=None, combine=True, keep_blocks=False, only=None):
        """only: names of the cell variables to keep (None: all of them)."""
        self.basename, self.dt, self.file_id = basename, float(dt), file_id
        self.variables, self.p0, self.species = variables, p0, species
        self.only = only
        self.combine, self.keep_blocks = combine, keep_blocks
        self.next_time = 0.0
        self.file_number = 0
        self.written = []

    def due(self, time, tlim, final=False):
        return final or time >= self.next_time or time >= tlim

    def write(self, source, time):
        blocks = _blocks_of(source)
        mesh_n = {1: blocks[0][0].nx1,
                  2: max(o[1] + c.nx2 for c, _, _, o in blocks),
                  3: max(o[2] + c.nx3 for c, _, _, o in blocks)}
        paths = []
        for gid, (cfg, x1f, w, off) in enumerate(blocks):
            dec = {d: (mesh_n[d], off[d - 1]) for d in (1, 2, 3)}
            path = block_filename(self.basename, gid, self.file_id, self.file_number)
            fields = cell_fields(cfg, w, self.variables, self.p0, self.species)
            if self.only is not None:
                fields = {k: v for k, v in fields.items() if k in self.only}
            write_file(path, coordinates(cfg, x1f), fields, time, dec, len(blocks))
            paths.append(path)
        out = paths
        if self.combine:
            out = [combine_blocks(self.basename, self.file_id, self.file_number,
                                  remove=not self.keep_blocks)]
        self.written += out
        self.file_number += 1
        self.next_time += self.dt
        return out


def combine_blocks(basename, file_id, number, remove=False):
    """Join the per-block files of one output into the whole-domain file,
    placing every block by the domain_decomposition of its coordinates
    (the job of mppnccombine in NetcdfOutput::CombineBlocks).  Returns the
    combined file's path."""
    pattern = f"{glob.escape(basename)}.block*.{glob.escape(file_id)}.{number:05d}.nc"
    rx = re.compile(re.escape(basename) + r"\.block(\d+)\.")
    paths = sorted(glob.glob(pattern), key=lambda s: int(rx.match(s).group(1)))
    if not paths:
        raise FileNotFoundError(pattern)
    parts = []
    for p in paths:
        with netcdf_file(p, "r", mmap=False) as f:
            dec = {d: f.variables[f"x{d}"].domain_decomposition.copy() for d in (1, 2, 3)}
            coords = {k: f.variables[k][:].copy() for k in f.variables if re.fullmatch(r"x\df?", k)}
            fields = {k: f.variables[k][0].copy() for k in f.variables
                      if k not in coords and k != "time"}
            units = {k: (getattr(f.variables[k], "long_name", b""),
                         getattr(f.variables[k], "units", b"")) for k in fields}
            time = float(f.variables["time"][0])
            order = [k for k in f.variables if k in fields]
        parts.append((dec, coords, fields))
    mesh_n = {d: int(parts[0][0][d][1]) for d in (1, 2, 3)}
    coords = {}
    for d in (1, 2, 3):
        c = np.zeros(mesh_n[d], dtype=np.float32)
        cf = np.zeros(mesh_n[d] + 1, dtype=np.float32)
        for dec, co, _ in parts:
            a, b = int(dec[d][2]) - 1, int(dec[d][3])
            c[a:b] = co[f"x{d}"]
            if f"x{d}f" in co:
                cf[a:b + 1] = co[f"x{d}f"]
        coords[f"x{d}"], coords[f"x{d}f"] = c, cf
    fields = {}
    for k in order:
        g = np.zeros((mesh_n[1], mesh_n[2], mesh_n[3]), dtype=np.float32)
        for dec, _, fl in parts:
            s = tuple(slice(int(dec[d][2]) - 1, int(dec[d][3])) for d in (1, 2, 3))
            g[s] = fl[k]
        fields[k] = g
    out = combined_filename(basename, file_id, number)
    write_file(out, coords, fields, time, None, len(paths))
    with netcdf_file(out, "a", mmap=False) as f:
        for k, (ln, un) in units.items():
            if ln:
                f.variables[k].long_name = ln
            if un:
                f.variables[k].units = un
    if remove:
        for p in paths:
            os.remove(p)
    return out


def join_records(paths, out):
    """One file holding the single time records of `paths` in order (the
    reference's outputs of one run joined along time, as ncrcat does), so a
    check can index the record of an output number."""
    with netcdf_file(paths[0], "r", mmap=False) as f0:
        dims = {k: v for k, v in f0.dimensions.items()}
        meta = {k: (f0.variables[k].dimensions, f0.variables[k].typecode(),
                    {a: getattr(f0.variables[k], a) for a in f0.variables[k]._attributes})
                for k in f0.variables}
        static = {k: f0.variables[k][:].copy() for k in f0.variables
                  if "time" not in f0.variables[k].dimensions}
    with netcdf_file(out, "w", version=1) as g:
        for k, n in dims.items():
            g.createDimension(k, n)
        for k, (d, tc, attrs) in meta.items():
            v = g.createVariable(k, tc, d)
            for a, val in attrs.items():
                setattr(v, a, val)
            if k in static:
                v[:] = static[k]
        for r, p in enumerate(paths):
            with netcdf_file(p, "r", mmap=False) as f:
                for k, (d, _, _) in meta.items():
                    if "time" in d:
                        g.variables[k][r] = f.variables[k][0]
    return out


def read_variable(path, name):
    with netcdf_file(path, "r", mmap=False) as f:
        return f.variables[name][:].copy()


def l2_difference(path1, path2, name, index):
    """sqrt(sum((a2 - a1)^2)) over variable `name`[index] of two files."""
    a = read_variable(path1, name)[index].astype(np.float64)
    b = read_variable(path2, name)[index].astype(np.float64)
    if a.shape != b.shape:
        raise ValueError(f"{name}{list(a.shape)} and {name}{list(b.shape)} differ in shape")
    return float(np.sqrt(np.sum((b - a) * (b - a))))


def check(case, path1, path2):
    """The example's regression test: returns the L2 norm when it is below
    the example's threshold, else raises ValueError."""
    name, index, limit = CHECKS[case]
    diff = l2_difference(path1, path2, name, index)
    if not diff < limit:
        raise ValueError(f"ERROR: {case} test failed. L2-norm is {diff:.2g}")
    return diff


def main(argv=None):
    argv = sys.argv[1:] if argv is None else argv
    if len(argv) != 3 or argv[0] not in CHECKS:
        print(f"usage: python -m canoe_b200.output {{{','.join(CHECKS)}}} case1.nc case2.nc",
              file=sys.stderr)
        return 2
    diff = check(*argv)
    print(f"### {argv[0]} test passed (L2-norm {diff:.3g}). ###")
    return 0


if __name__ == "__main__":
    sys.exit(main())
