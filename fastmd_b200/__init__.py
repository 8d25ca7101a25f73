"""fastmd_b200: bead-spring polymer MD per-step path on NVIDIA B200.

Python bindings over the C ABI in include/fastmd.h (libfastmd_b200.so, built
in-tree by ``make -C fastmd_b200/csrc``).  There is no Python or CPU
implementation of the path behind these bindings: if the shared library is
missing, importing this package raises.

The objects mirror the reference fastMD's user-facing interface: a simulation
is created from the same run.conf text (src/io/config.cpp:32-127) and a LAMMPS
data file, a generated melt, or in-memory arrays; thermo and rg values are the
ones behind the reference's output columns (src/analysis/thermo.cu:192,
src/analysis/rg.cu:127).
"""
from __future__ import annotations

from ._lib import (  # noqa: F401
    FMD_FORM_MIXED,
    FMD_FORM_PLAIN_FP64,
    FMD_LANGEVIN,
    FMD_NPT_NH,
    FMD_NVT_NH,
    Batch,
    FastMDError,
    MeltSpec,
    Server,
    ServerPool,
    Simulation,
    SystemDesc,
    ThermoRow,
    Trajectory,
    format_rg_row,
    format_thermo_row,
    generate_melt,
    lib,
    lib_path,
    parse_run_conf,
    partition_replicas,
    read_lammps_data,
    read_pair_table,
    run_conf_tables,
    read_trajectory,
    write_lammps_data,
)

__version__ = "0.1.0"
