"""The C ABI library builds for sm_100a, loads without a GPU, exports every
function include/pbpic.h declares, and its structs match the Python views
(CPU; no compute calls)."""
import ctypes
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "pbpic.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(pbpic_\w+)\s*\(", text)))


def test_header_declares_the_step_boundary():
    names = declared_functions()
    for need in ("pbpic_create", "pbpic_destroy", "pbpic_push", "pbpic_fieldsolve", "pbpic_sort", "pbpic_step",
                 "pbpic_energies", "pbpic_gauss_residual", "pbpic_load_particles_f32", "pbpic_store_particles_f32",
                 "pbpic_load_fields_f64", "pbpic_store_denjr_f64", "pbpic_last_error"):
        assert need in names


def test_library_exports_every_declared_symbol():
    from pbpic_b200 import build
    lib_path = build.build()
    lib = ctypes.CDLL(lib_path)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_signatures_cover_the_header():
    from pbpic_b200 import _lib
    declared = set(declared_functions()) - {"pbpic_last_error"}
    assert declared == set(_lib.SIGNATURES)


def test_struct_layouts_match_c(tmp_path):
    from pbpic_b200 import _lib
    src = tmp_path / "sz.c"
    src.write_text(
        '#include <stdio.h>\n#include <stddef.h>\n#include "pbpic.h"\n'
        "int main(void){printf(\"%zu %zu %zu %zu %zu %zu\\n\", sizeof(pbpic_config), sizeof(pbpic_loader),"
        " sizeof(pbpic_particle_f32), sizeof(pbpic_particle_f64), offsetof(pbpic_config, capacity),"
        " offsetof(pbpic_loader, seed));return 0;}\n")
    exe = tmp_path / "sz"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), "-o", str(exe), str(src)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    assert got == [ctypes.sizeof(_lib.Config), ctypes.sizeof(_lib.Loader), _lib.PARTICLE_F32.itemsize,
                   _lib.PARTICLE_F64.itemsize, _lib.Config.capacity.offset, _lib.Loader.seed.offset]


def test_create_reports_errors_without_crashing():
    """Invalid configurations are rejected with a message before any device work."""
    import pbpic_b200
    from pbpic_b200 import configs
    cfg, _ = configs.uniform_c1(mx=8, my=8)
    bad = dict(cfg, mx=1)
    with pytest.raises(pbpic_b200.PbpicError) as e:
        pbpic_b200.Simulation(**bad)
    assert "mx" in str(e.value)
    with pytest.raises(pbpic_b200.PbpicError) as e:
        pbpic_b200.Simulation(**dict(cfg, dt=cfg["dt"] * 4))
    assert "CFL" in str(e.value)


def test_batch_create_rejects_bad_domains_before_device_work():
    """The batched form takes FP32 mixed domains with mx >= 3 (and my >= 3 with periodic y)."""
    import pbpic_b200
    from pbpic_b200 import _lib, configs
    from pbpic_b200.batch import Batch
    cfg, ld = configs.two_stream(8, 8, 4, seed=1)
    with pytest.raises(pbpic_b200.PbpicError) as e:
        Batch([(cfg, ld), (dict(cfg, mx=2), ld)])
    assert "mx >= 3" in str(e.value)
    lib = _lib.lib()
    cfgs = (_lib.Config * 1)()
    for k, v in cfg.items():
        setattr(cfgs[0], k, v)
    cfgs[0].precision = _lib.FP64_PLAIN
    loaders = (_lib.Loader * 1)()
    out = ctypes.c_void_p()
    assert lib.pbpic_batch_create(cfgs, loaders, 1, ctypes.byref(out)) == -1
    assert b"FP32" in lib.pbpic_last_error()
    assert lib.pbpic_batch_create(cfgs, loaders, 0, ctypes.byref(out)) == -1


def test_fortran_module_binds_exported_symbols():
    """Every bind(c) name in the Fortran interface module is a function the
    library exports (the module cannot be compiled here: no Fortran compiler)."""
    from pbpic_b200 import build
    lib = ctypes.CDLL(build.build())
    src = open(os.path.join(ROOT, "pbpic_b200", "fortran", "pbpic_gpu.f90")).read()
    names = set(re.findall(r'bind\(c,\s*name="(pbpic_\w+)"\)', src))
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) <= set(declared_functions()) | {"pbpic_last_error"}


FORTRAN = os.path.join(ROOT, "pbpic_b200", "fortran", "pbpic_gpu.f90")
_FKIND = {"c_int32_t": ("i", 4), "c_int64_t": ("i", 8), "c_double": ("f", 8), "c_float": ("f", 4)}


def fortran_records(text):
    """name -> [(field, (kind letter, bytes))] of every `type, bind(c)` block."""
    out = {}
    for name, body in re.findall(r"type, bind\(c\) :: (\w+)\n(.*?)end type", text, flags=re.S):
        fields = []
        for line in body.splitlines():
            line = line.split("!")[0].strip()
            if "::" not in line:
                continue
            decl, names = line.split("::")
            kind = _FKIND[re.search(r"\((c_\w+)\)", decl).group(1)]
            fields += [(n.strip(), kind) for n in names.split(",")]
        out[name] = fields
    return out


def _ctypes_kind(t):
    return ("f" if t in (ctypes.c_double, ctypes.c_float) else "i", ctypes.sizeof(t))


def test_fortran_module_matches_the_header():
    """The Fortran module (not compiled here: no Fortran compiler) binds only
    functions the header declares, and its records list the C structs' fields
    in order with the same kinds and sizes."""
    from pbpic_b200 import _lib
    text = open(FORTRAN).read()
    names = re.findall(r'bind\(c,\s*name="(pbpic_\w+)"\)', text)
    assert names and set(names) <= set(declared_functions())
    recs = fortran_records(text)
    rename = {"lambda": "lambda_"}
    for fname, cls in (("pbpic_config", _lib.Config), ("pbpic_loader", _lib.Loader)):
        got = [(rename.get(n, n), k) for n, k in recs[fname]]
        assert got == [(n, _ctypes_kind(t)) for n, t in cls._fields_], fname
    for fname, dt in (("c_particle", _lib.PARTICLE_F32), ("c_particle_f64", _lib.PARTICLE_F64)):
        assert [(n, k) for n, k in recs[fname]] == [(n, (dt[n].kind, dt[n].itemsize)) for n in dt.names], fname
