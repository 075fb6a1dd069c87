"""CPU tests of the library's host side: the C-ABI library loads and exports every
function include/rbc.h declares, its Galerkin tables match the reference's golden
vectors, and invalid construction parameters are rejected without a GPU call."""
import ctypes
import os
import re

import numpy as np
import pytest

import sdc_b200

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, "tests", "golden")


def declared_functions():
    hdr = open(os.path.join(ROOT, "include", "rbc.h")).read()
    hdr = re.sub(r"/\*.*?\*/", "", hdr, flags=re.S)
    return sorted(set(re.findall(r"\b(rbc_[a-z_0-9]+)\s*\(", hdr)))


def test_library_exports_every_declared_symbol():
    lib = sdc_b200.lib()
    names = declared_functions()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(sdc_b200.EXPORTS)


@pytest.mark.parametrize("L", [4, 8, 12])
@pytest.mark.parametrize("name", ["Iac", "Ia1", "Ia2", "Ibbb", "Ibb1", "Ib11", "I111", "Iabc", "Iac1",
                                  "Iaab", "Iaa1", "Iab2", "Ia12", "lambda"])
def test_library_tables_match_reference_golden(L, name):
    ref = np.load(os.path.join(GOLD, f"coeff_L{L}.npz"))[name]
    got = sdc_b200.galerkin_table(L, name)
    assert got.shape == ref.shape
    assert np.abs(got - ref).max() <= 1e-13 * np.abs(ref).max()


def test_unknown_table_rejected():
    with pytest.raises(sdc_b200.RBCError):
        sdc_b200.galerkin_table(4, "nope")


def test_status_strings():
    lib = sdc_b200.lib()
    for s in range(8):
        assert lib.rbc_status_string(s)


def test_invalid_params_rejected_before_any_device_work():
    # nx = 100 is not 2^a 3^b: refused by argument checks (no CUDA call is made)
    with pytest.raises(sdc_b200.RBCError) as e:
        sdc_b200.Solver(100, 64, 4, 8.0, 8.0, 2000.0, 1.0, 1e-3)
    assert e.value.status == 1
    with pytest.raises(sdc_b200.RBCError) as e:
        sdc_b200.Solver(64, 64, 4, 8.0, 8.0, 2000.0, -1.0, 1e-3)
    assert e.value.status == 1
    with pytest.raises(sdc_b200.RBCError) as e:
        sdc_b200.Solver(64, 64, 7, 8.0, 8.0, 2000.0, 1.0, 1e-3)
    assert e.value.status == 6


@pytest.mark.parametrize("kw", [
    dict(field_ops=("freeze",), penalization=(-0.5, "rectangle")),  # negative eta
    dict(penalization=(float("inf"), "circle")),
    dict(mean_F=float("nan")),
    dict(n_tracers=100, tracer_sets=3),                              # sets must divide the tracers
    dict(n_tracers=0, tracer_sets=2),
    dict(tracer_sets=-1),
])
def test_invalid_optional_physics_params_rejected_before_any_device_work(kw):
    with pytest.raises(sdc_b200.RBCError) as e:
        sdc_b200.Solver(64, 64, 4, 8.0, 8.0, 2000.0, 1.0, 1e-3, **kw)
    assert e.value.status == 1


def test_params_struct_matches_header_layout():
    """The ctypes mirror of rbc_params has the header's fields in the header's order."""
    hdr = open(os.path.join(ROOT, "include", "rbc.h")).read()
    body = hdr[hdr.index("typedef struct {\n    int nx;"):hdr.index("} rbc_params;")]
    names = re.findall(r"^\s+(?:unsigned long long|double|int)\s+([\w, ]+);", body, re.M)
    fields = [n.strip() for group in names for n in group.split(",")]
    assert fields == [f[0] for f in sdc_b200._Params._fields_]


def test_cli_driver_rejects_unknown_penalization_mask(tmp_path):
    import subprocess
    exe = os.path.join(os.path.dirname(sdc_b200.LIB_PATH), "rbc_run")
    r = subprocess.run([exe, "-nmodes", "32", "32", "3", "-clength", "8", "8", "-ra", "3000", "-pr", "1",
                        "-dt", "1e-3", "-t", "0.001", "-penalized", "hexagon", "-dir", str(tmp_path)],
                       capture_output=True, text=True, timeout=60)
    assert r.returncode == 2 and "hexagon" in r.stderr


def test_cli_driver_usage_and_le_count_mismatch(tmp_path):
    import subprocess
    exe = os.path.join(os.path.dirname(sdc_b200.LIB_PATH), "rbc_run")
    r = subprocess.run([exe, "-h"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0 and "usage" in r.stdout
    r = subprocess.run([exe, "-nmodes", "32", "32", "3", "-clength", "8", "8", "-ra", "3000", "-pr", "1",
                        "-dt", "1e-3", "-t", "0.001", "-npart", "16", "-le_count", "3", "-le", "1", "0.1",
                        "-dir", str(tmp_path)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 2 and "-le" in r.stderr


def test_header_is_plain_c99_and_links(tmp_path):
    """include/rbc.h compiles as C99 and every declared function links against the library
    with C linkage (the program is built, not run)."""
    import subprocess
    names = declared_functions()
    src = tmp_path / "use.c"
    src.write_text('#include "rbc.h"\ntypedef void (*fn)(void);\nint main(void) {\n    volatile fn t[] = {\n' +
                   "".join(f"        (fn)&{n},\n" for n in names) + "    };\n    return t[0] == 0;\n}\n")
    lib_dir = os.path.dirname(sdc_b200.LIB_PATH)
    r = subprocess.run(["gcc", "-std=c99", "-Wall", "-pedantic", "-Werror", "-I", os.path.join(ROOT, "include"),
                        str(src), "-L", lib_dir, "-lsdc_b200", "-o", str(tmp_path / "use")],
                       capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert len(names) == len(sdc_b200.EXPORTS)
