"""The `fastmd <run.conf>` program's argument and error handling, and the
host helpers it is built on (no GPU needed: every case below fails or
finishes before a device is touched).

Follows src/main.cu:24-36 (usage message, exit status 1) and
src/io/config.cpp (deprecated keys raise with the reference's messages);
restart names follow io/lammps_data.cpp:255-267."""
import ctypes as C
import os
import subprocess

import pytest

import fastmd_b200 as fm

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "fastmd_b200", "bin", "fastmd")


def _run(args, cwd):
    assert os.path.exists(CLI), "fastmd_b200/bin/fastmd is not built (make -C fastmd_b200/csrc)"
    return subprocess.run([CLI] + args, cwd=cwd, capture_output=True, text=True, timeout=60)


def test_usage_without_arguments(tmp_path):
    out = _run([], tmp_path)
    assert out.returncode == 1 and "Usage:" in out.stderr and "<config_file>" in out.stderr


def test_missing_config_file(tmp_path):
    out = _run(["nope.conf"], tmp_path)
    assert out.returncode == 1 and "cannot open config file nope.conf" in out.stderr


def test_unknown_option(tmp_path):
    out = _run(["--fast", "x.conf"], tmp_path)
    assert out.returncode == 1 and "unknown option --fast" in out.stderr


@pytest.mark.parametrize("key,msg", [
    ("temperature 1.0", "'temperature' is deprecated. Use 'nvt_langevin T_start T_stop Tdamp [seed]' instead."),
    ("gamma 1.0", "'gamma' is deprecated. Use 'nvt_langevin T_start T_stop Tdamp [seed]' instead."),
    ("seed 5", "'seed' as a standalone key is deprecated."),
])
def test_deprecated_keys_fail_like_the_reference(tmp_path, key, msg):
    (tmp_path / "run.conf").write_text(f"ntypes 1\nrc 2.5\nskin 0.3\ndt 0.001\nnsteps 10\n{key}\n")
    out = _run(["run.conf"], tmp_path)
    assert out.returncode == 1 and msg in out.stderr


def test_config_errors_exit_one(tmp_path):
    (tmp_path / "run.conf").write_text("ntypes 1\nrc 2.5\nskin 0.3\ndt 0.001\nnsteps 10\nnvt_langevin 1 1 0\n")
    out = _run(["run.conf"], tmp_path)
    assert out.returncode == 1 and "Tdamp must be > 0 for nvt_langevin" in out.stderr


def test_run_conf_outputs():
    lib = fm.lib()

    class Spec(C.Structure):
        _fields_ = [("nsteps", C.c_int64), ("ensemble", C.c_int32), ("thermo_on", C.c_int32),
                    ("thermo_freq", C.c_int32), ("rg_on", C.c_int32), ("rg_freq", C.c_int32),
                    ("stress_on", C.c_int32), ("stress_freq", C.c_int32), ("dump_freq", C.c_int32),
                    ("restart_freq", C.c_int32), ("thermo_file", C.c_char * 256), ("rg_file", C.c_char * 256),
                    ("stress_file", C.c_char * 256), ("restart_file", C.c_char * 256),
                    ("data_file", C.c_char * 256), ("forces_dump_file", C.c_char * 256)]

    text = (b"ntypes 1\nrc 2.5\nskin 0.3\ndt 0.001\nnsteps 5000\nnvt_nh 1 1 0.5\nthermo 1 100 th.dat\n"
            b"rg 1 200 rg.dat\nrestart 1000 out/restart.data\ndump_freq 250\nstress 1 10 s.dat\n"
            b"lammps_data_file melt.data\n")
    s = Spec()
    assert lib.fmd_run_conf_outputs(text, C.byref(s)) == 0
    assert (s.nsteps, s.ensemble, s.thermo_on, s.thermo_freq, s.rg_freq, s.dump_freq, s.restart_freq,
            s.stress_freq) == (5000, 1, 1, 100, 200, 250, 1000, 10)
    assert s.thermo_file == b"th.dat" and s.restart_file == b"out/restart.data" and s.data_file == b"melt.data"
    s2 = Spec()
    assert lib.fmd_run_conf_outputs(b"ntypes 1\nrc 2.5\nskin 0.3\ndt 0.001\nnvt_langevin 1 1 1\n", C.byref(s2)) == 0
    assert s2.restart_freq == -1 and s2.thermo_on == 0   # no restart key: no restart files (main.cu:738)


@pytest.mark.parametrize("base,step,want", [("restart.data", 500, "restart_500.data"),
                                            ("restart.data", -1, "restart_final.data"),
                                            ("out/run.lmp", 20, "out/run_20.lmp"),
                                            ("restart", 7, "restart_7"), ("restart", -1, "restart_final")])
def test_restart_filenames(base, step, want):
    buf = C.create_string_buffer(256)
    assert fm.lib().fmd_restart_filename(base.encode(), C.c_int64(step), buf, C.c_size_t(256)) == 0
    assert buf.value.decode() == want
