"""C-ABI checks that need no GPU: exports, struct layout, validation, sizing."""
import ctypes as C
import re
import subprocess
import textwrap
from pathlib import Path

import numpy as np
import pytest

import stochasticphysics_b200 as sp
from stochasticphysics_b200 import _abi, provider
from stochasticphysics_b200.lib import LIB_PATH, SYMBOLS, load

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "stophys_b200.h"


def declared_symbols():
    return sorted(set(re.findall(r"^SP_API [^(]*?\b(sp_\w+)\(", HEADER.read_text(), flags=re.M)))


def test_library_exports_every_declared_symbol():
    lib = load()
    names = declared_symbols()
    assert len(names) >= 20
    assert sorted(SYMBOLS) == names
    for n in names:
        assert hasattr(lib, n), n
    out = subprocess.run(["nm", "-D", "--defined-only", str(LIB_PATH)], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (sp_\w+)", out))
    assert set(names) <= exported
    # nothing but the ABI is exported under the sp_ prefix
    assert exported == set(names)


def test_abi_version_and_dims():
    lib = load()
    header_version = int(re.search(r"#define SP_ABI_VERSION (\d+)u", HEADER.read_text()).group(1))
    assert lib.sp_abi_version() == _abi.ABI_VERSION == header_version
    for prob, dims in _abi.DIMS.items():
        a, b, c = C.c_int32(), C.c_int32(), C.c_int32()
        assert lib.sp_query_dims(int(prob), C.byref(a), C.byref(b), C.byref(c)) == 0
        assert (a.value, b.value, c.value) == dims
    assert lib.sp_query_dims(9, None, None, None) == int(sp.Status.INVALID_ARG)


def test_ctypes_layout_matches_c(tmp_path):
    """offsetof/sizeof of the public structs, compiled from the header, equal the ctypes mirror."""
    fields = {
        "sp_ensemble_desc": _abi.sp_ensemble_desc, "sp_particles": _abi.sp_particles, "sp_field_desc": _abi.sp_field_desc,
        "sp_problem_settings": _abi.sp_problem_settings, "sp_result": _abi.sp_result, "sp_stats": _abi.sp_stats,
        "sp_server_config": _abi.sp_server_config, "sp_launch_config": _abi.sp_launch_config,
        "sp_dist": _abi.sp_dist, "sp_particle_template": _abi.sp_particle_template,
        "sp_provider_desc": _abi.sp_provider_desc,
    }
    lines = []
    for cname, cls in fields.items():
        lines.append(f'printf("{cname} sizeof %zu\\n", sizeof({cname}));')
        for fname, _ in cls._fields_:
            lines.append(f'printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    src = tmp_path / "layout.c"
    src.write_text(textwrap.dedent(f"""
        #include <stdio.h>
        #include <stddef.h>
        #include "stophys_b200.h"
        int main(void) {{ {' '.join(lines)} return 0; }}
    """))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c99", "-I", str(HEADER.parent), str(src), "-o", str(exe)], check=True)
    got = {}
    for line in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.splitlines():
        s, f, v = line.split()
        got[(s, f)] = int(v)
    for cname, cls in fields.items():
        assert got[(cname, "sizeof")] == C.sizeof(cls), cname
        for fname, _ in cls._fields_:
            assert got[(cname, fname)] == getattr(cls, fname).offset, (cname, fname)


def _validate(spec):
    h = _abi.DescHolder(spec)
    rc = load().sp_validate(h.byref())
    msg = load().sp_last_error().decode()
    return rc, msg


def test_validate_accepts_the_workloads():
    for spec in (provider.neel_relaxation(n=10, steps=1000), provider.brown_neel_relaxation(n=10, steps=2000),
                 provider.cubic_implicit(n=10, steps=2000)):
        assert _validate(spec)[0] == 0


@pytest.mark.parametrize("mutate,status,text", [
    (dict(oversampling=0), sp.Status.INVALID_ARG, "oversampling"),
    (dict(number_of_steps=5, oversampling=10), sp.Status.INVALID_ARG, "number_of_steps"),
    (dict(timestep=0.0), sp.Status.INVALID_ARG, "timestep"),
    (dict(timestep=float("nan")), sp.Status.INVALID_ARG, "timestep"),
    (dict(temperature=-1.0), sp.Status.INVALID_ARG, "temperature"),
    (dict(max_iteration=0, solver=sp.Solver.Implicit_Midpoint), sp.Status.INVALID_ARG, "max_iteration"),
    (dict(noise=sp.Noise.Injected), sp.Status.INVALID_ARG, "injected_dw"),
])
def test_validate_rejects_malformed(mutate, status, text):
    import dataclasses
    spec = dataclasses.replace(provider.neel_relaxation(n=8, steps=1000), **mutate)
    rc, msg = _validate(spec)
    assert rc == int(status)
    assert text in msg


def test_validate_unsupported_combination():
    import dataclasses
    spec = dataclasses.replace(provider.brown_neel_relaxation(n=8, steps=2000), solver=sp.Solver.Implicit_Midpoint)
    rc, msg = _validate(spec)
    assert rc == int(sp.Status.UNSUPPORTED_COMBO)
    assert "Jacobian" in msg


def test_validate_brown_needs_hydrodynamics():
    import dataclasses
    spec = dataclasses.replace(provider.brown_neel_relaxation(n=8, steps=2000), hydrodynamic_radius=None)
    rc, msg = _validate(spec)
    assert rc == int(sp.Status.INVALID_ARG) and "hydrodynamic" in msg


def test_footprint_scales_with_particles():
    small = sp.Context.footprint(provider.brown_neel_relaxation(n=1000, steps=20000))
    big = sp.Context.footprint(provider.brown_neel_relaxation(n=64000, steps=20000))
    assert 0 < small < big
    # FP32 state is smaller than FP64 state
    import dataclasses
    s32 = sp.Context.footprint(dataclasses.replace(provider.brown_neel_relaxation(n=64000, steps=20000),
                                                   precision=sp.Precision.FP32))
    assert s32 < big


def test_create_without_device_fails_loudly():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a CUDA device is present")
    except ImportError:
        pass
    with pytest.raises(sp.SPError) as ei:
        sp.Context(0)
    assert ei.value.status in (int(sp.Status.NO_DEVICE), int(sp.Status.CUDA))


def test_server_entry_points_refuse_null_arguments():
    """The server calls check their arguments before touching a device."""
    lib = load()
    ids = (C.c_uint64 * 2)()
    assert lib.sp_server_submit_many(None, None, 2, ids) == int(sp.Status.INVALID_ARG)
    assert "NULL" in lib.sp_last_error().decode()
    assert lib.sp_server_submit(None, None, None) == int(sp.Status.INVALID_ARG)
    assert lib.sp_server_poll(None, 1, None) == int(sp.Status.INVALID_ARG)
