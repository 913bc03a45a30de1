"""Output and restart files of the coupler (coupler.h:533-723 of the
reference) with the dycore's write and restart hooks (dynamics_rk.h:1191-1242).

The reference writes NetCDF through PnetCDF (64-bit data format); this image
has no NetCDF library, so files are written with ``scipy.io.netcdf_file`` in
the 64-bit-offset classic format, which every NetCDF reader opens.  The
variables, dimensions and types are the reference's:

* dimensions ``x``, ``y``, ``z``, ``t`` (1);
* ``x``, ``y``, ``z`` cell-centre coordinates, ``etime``, ``file_counter``;
* ``density_dry``, ``uvel``, ``vvel``, ``wvel``, ``temperature`` and every
  tracer, (z, y, x), float32 -- or float64 with the coupler option
  ``output_f64`` set, which makes a restart exact (the reference's float
  restart is not);
* registered output variables (``Coupler.register_output_variable``);
* whatever the registered write modules add (the dycore: ``z_halo``,
  ``hy_*_cells`` float32 -- float64 with ``output_f64`` --, ``density_pert``,
  ``theta_pert``, ``pressure_pert`` float64).

``overwrite_with_restart`` reads the state back from the file named by the
option ``restart_file`` and runs the registered restart modules.
"""
from __future__ import annotations

import numpy as np
from scipy.io import netcdf_file

DIMS_COLUMN, DIMS_SURFACE, DIMS_3D = 1, 2, 3
_DIMNAMES = {DIMS_COLUMN: ("z",), DIMS_SURFACE: ("y", "x"), DIMS_3D: ("z", "y", "x")}


def _host(a):
    """numpy view of a coupler array (numpy or torch tensor)."""
    if isinstance(a, np.ndarray):
        return a
    return a.detach().cpu().numpy()


def _assign(dst, src):
    """dst[...] = src for a numpy or torch destination."""
    if isinstance(dst, np.ndarray):
        dst[...] = src
    else:
        import torch
        dst.copy_(torch.from_numpy(np.ascontiguousarray(src, dtype=np.float64)).to(dst.dtype))


class NetCDF:
    """The subset of yakl::SimplePNetCDF the output modules use, over
    scipy.io.netcdf_file."""

    def __init__(self, path, mode):
        self.f = netcdf_file(path, mode, version=2, mmap=False) if mode == "w" else \
            netcdf_file(path, mode, mmap=False)

    def create_dim(self, name, n):
        self.f.createDimension(name, n)

    def create_var(self, name, dims, dtype):
        return self.f.createVariable(name, np.dtype(dtype), tuple(dims))

    def write(self, data, name):
        v = self.f.variables[name]
        v[...] = np.asarray(data, dtype=v.data.dtype).reshape(v.shape)

    def read(self, name):
        """The variable as a native-endian array (NetCDF stores big-endian)."""
        d = self.f.variables[name].data
        return np.array(d, dtype=d.dtype.newbyteorder("="), copy=True)

    def has(self, name):
        return name in self.f.variables

    def close(self):
        self.f.close()


def write_output_file(coupler, prefix, verbose=False):
    """coupler.h:533-649: writes ``<prefix>_<counter:08d>.nc`` and advances
    the coupler's file counter; returns the file name."""
    nx, ny, nz = coupler.get_nx(), coupler.get_ny(), coupler.get_nz()
    dx, dy, dz = coupler.get_dx(), coupler.get_dy(), coupler.get_dz()
    state_type = np.float64 if coupler.get_option("output_f64", False) else np.float32
    fname = "%s_%08d.nc" % (prefix, coupler.file_counter)
    nc = NetCDF(fname, "w")
    nc.create_dim("x", nx)
    nc.create_dim("y", ny)
    nc.create_dim("z", nz)
    nc.create_dim("t", 1)
    for name, n, d in (("x", nx, dx), ("y", ny, dy), ("z", nz, dz)):
        nc.create_var(name, (name,), np.float32)
        nc.write((np.arange(n) + 0.5) * d, name)
    nc.create_var("etime", ("t",), np.float32)
    nc.write([coupler.get_option("elapsed_time", 0.0)], "etime")
    nc.create_var("file_counter", ("t",), np.int32)
    nc.write([coupler.file_counter], "file_counter")
    fields = [("density_dry", "density_dry"), ("uvel", "uvel"), ("vvel", "vvel"), ("wvel", "wvel"),
              ("temperature", "temp")] + [(n, n) for n in coupler.get_tracer_names()]
    for var, entry in fields:
        nc.create_var(var, ("z", "y", "x"), state_type)
        nc.write(_host(coupler.get(entry)), var)
    for name, dims, dtype in coupler.output_vars:
        out_type = np.float32 if np.issubdtype(np.dtype(dtype), np.floating) else dtype
        nc.create_var(name, _DIMNAMES[dims], out_type)
        nc.write(_host(coupler.get(name)), name)
    for f in coupler.write_output_modules:
        f(coupler, nc)
    nc.close()
    coupler.file_counter += 1
    if verbose:
        print("*** Output/restart file written *** -->", fname)
    return fname


def overwrite_with_restart(coupler):
    """coupler.h:653-723: state, tracers and registered output variables from
    the file named by the option ``restart_file``, then the registered
    restart modules; sets ``elapsed_time`` and the file counter."""
    nc = NetCDF(coupler.get_option("restart_file"), "r")
    coupler.set_option("elapsed_time", float(nc.read("etime")[0]))
    coupler.file_counter = int(nc.read("file_counter")[0])
    fields = [("density_dry", "density_dry"), ("uvel", "uvel"), ("vvel", "vvel"), ("wvel", "wvel"),
              ("temperature", "temp")] + [(n, n) for n in coupler.get_tracer_names()]
    for var, entry in fields:
        _assign(coupler.get(entry), nc.read(var).astype(np.float64))
    for name, _, _ in coupler.output_vars:
        dst = coupler.get(name)
        _assign(dst, nc.read(name))
    for f in coupler.restart_modules:
        f(coupler, nc)
    nc.close()
    coupler.file_counter += 1


def dycore_write_hook(handle_of):
    """The dycore's write module (dynamics_rk.h:1193-1233): the hydrostatic
    cell profiles (float32, dimension z_halo) and the FP64 density, theta and
    pressure perturbations of the coupler state, computed on the GPU."""

    def hook(coupler, nc):
        h = handle_of(coupler)
        nzh = coupler.get_nz() + 2 * 4
        nc.create_dim("z_halo", nzh)
        # float32 as the reference stores them; with output_f64 the handle's
        # own profiles (FP64 in the FP64 build), so that a restart is exact.
        f64 = coupler.get_option("output_f64", False)
        cells, _ = h.get_hydrostasis()
        for name, prof in zip(("hy_dens_cells", "hy_theta_cells", "hy_pressure_cells"), cells):
            nc.create_var(name, ("z_halo",), np.float64 if f64 else np.float32)
            nc.write(prof if f64 else _host(coupler.get(name)), name)
        arrays = [coupler.get(n) for n in ("density_dry", "uvel", "vvel", "wvel", "temp")]
        trc = [coupler.get(n) for n in coupler.get_tracer_names()]
        for name, data in zip(("density_pert", "theta_pert", "pressure_pert"), h.perturbations(*arrays, trc)):
            nc.create_var(name, ("z", "y", "x"), np.float64)
            nc.write(data, name)

    return hook


def dycore_restart_hook(handle_of):
    """The dycore's restart module (dynamics_rk.h:1235-1242): the hydrostatic
    cell profiles from the file; the handle recomputes its edge profiles."""

    def hook(coupler, nc):
        cells = [nc.read(n) for n in ("hy_dens_cells", "hy_theta_cells", "hy_pressure_cells")]
        for name, a in zip(("hy_dens_cells", "hy_theta_cells", "hy_pressure_cells"), cells):
            coupler.dm[name] = a.astype(np.float32)
        handle_of(coupler).set_hydrostasis(*[a.astype(np.float64) for a in cells])

    return hook
