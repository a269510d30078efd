"""CPU tests of the C ABI library: it loads, exports every function that
include/ldp.h declares, and its host-side pieces (.inp grammar, defaults)
behave like the reference's InputParser.  No kernel is launched."""
import ctypes as C
import os
import re

import pytest

import langevindynamicsforpcp_b200 as ldp
from langevindynamicsforpcp_b200 import _lib as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "ldp.h")
GOLDEN = os.path.join(ROOT, "tests", "golden", "inp")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(ldp_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_function():
    h = L.lib()
    names = declared_functions()
    assert len(names) >= 20
    for n in names:
        assert hasattr(h, n), n
        assert n in L.SIGNATURES, f"{n} has no ctypes signature"
    assert h.ldp_abi_version() == L.ABI_VERSION == 2


def test_status_strings():
    assert L.lib().ldp_status_string(0) == b"ok"
    assert L.lib().ldp_status_string(6) == b"parse error"


def quick_text():
    return open(os.path.join(GOLDEN, "quick_test__2.0_7.2_m1.0_1.00e-05.inp")).read()


def test_parse_quick_test_values():
    p = ldp.params_from_inp_text(quick_text())
    assert p.output_base == b"m1.0_t1.00e-05_0"
    assert p.overdamped == 1 and p.x0 == -2.9 and p.periodic_length == 5.8
    assert tuple(p.barrier_heights[0]) == (7.2, 2.0)
    assert p.barrier_half_width[0] == 0.65 and p.timestep == 1e-4 and p.tau == 1e-5
    assert p.number_of_steps == 3_000_000_000 and p.freq_save == 300_000
    assert p.fptcg == 1 and p.n_cg == 7 and list(p.cg_sizes[:7]) == [2, 3, 4, 5, 10, 100, 1000]
    assert p.random_seed == 123 and p.number_of_log_samples == 40
    assert p.write_x == 1 and p.write_restart == 1 and p.eq == 1 and p.eq_constant == 1.0


def test_parse_double_barrier_values():
    p = ldp.params_from_inp(os.path.join(GOLDEN, "CuIDB_double__2.0_7.2_m1.0_1.00e-05.inp"), ldp.MODEL_DOUBLE)
    assert tuple(p.barrier_heights[0]) == (3.4, 2.0) and tuple(p.barrier_heights[1]) == (7.2, 2.0)
    assert tuple(p.barrier_half_width) == (0.7, 0.65) and tuple(p.barrier_position) == (-1.42, -0.56)


def test_grammar_define_variables_continuation_for():
    base = quick_text().replace("X0                   -2.9", "")
    base = base.replace("TIMESTEP             0.0001", "TIMESTEP \\\n   0.0002")
    base = base.replace("FPTCG                true 1000", "FOR 0 3 1 %d I FPTCG true 7I")
    txt = "DEFINE @XX@ -1.5\nmyvar = 0.25\nX0 @XX@\n" + base.replace("BARRIERHALFWIDTH     0.65",
                                                                       "BARRIERHALFWIDTH myvar")
    p = ldp.params_from_inp_text(txt)
    assert p.x0 == -1.5 and p.barrier_half_width[0] == 0.25 and p.timestep == 2e-4
    assert list(p.cg_sizes[:p.n_cg]) == [2, 3, 4, 5, 10, 100, 70, 71, 72]


def test_grammar_include(tmp_path, monkeypatch):
    # INCLUDE paths are opened as written, relative to the working directory
    # (the reference's OpenInput, src/inputParser.cpp:311), not relative to
    # the including file: main.inp in inputs/ includes parts/part.inp, which
    # lies under the working directory.
    txt = quick_text()
    head, tail = txt[: len(txt) // 2], txt[len(txt) // 2:]
    cut = head.rfind("\n")
    head, tail = txt[:cut + 1], txt[cut + 1:]
    (tmp_path / "inputs").mkdir()
    (tmp_path / "parts").mkdir()
    (tmp_path / "parts" / "part.inp").write_text(tail)
    (tmp_path / "inputs" / "main.inp").write_text(head + "INCLUDE parts/part.inp\n")
    monkeypatch.chdir(tmp_path)
    p = ldp.params_from_inp("inputs/main.inp")
    q = ldp.params_from_inp_text(txt)
    assert bytes(p) == bytes(q)
    # the same name next to the including file is not what the reference opens
    monkeypatch.chdir(tmp_path / "inputs")
    with pytest.raises(Exception, match="can't open input file"):
        ldp.params_from_inp("main.inp")


def test_print_values_is_the_references_print_all_values(tmp_path):
    # `-p`: every option in option-table order, one "%-20s %3d %s" line per
    # occurrence (InputParser::PrintAllValues, src/inputParser.cpp:188-196),
    # on stderr; the FPTCG occurrences are numbered 0..n-1.
    path = os.path.join(GOLDEN, "quick_test__2.0_7.2_m1.0_1.00e-05.inp")
    entries = {}
    for ln in open(path):
        w = ln.split("#")[0].split()
        if not w:
            continue
        if w[0] not in entries:
            entries[w[0]] = []
        entries[w[0]].append(" ".join(w[1:]))
    exe = os.path.join(ROOT, "langevindynamicsforpcp_b200", "bin", "langevinDynamicsSingleBarrier")
    import subprocess
    r = subprocess.run([exe, "-i", path, "-p"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stderr
    lines = r.stderr.splitlines()
    parsed = []
    for l in lines:
        m = re.match(r"^(\S+) +(\d+) (.*)$", l)
        assert m, l
        key, idx, val = m.group(1), int(m.group(2)), m.group(3)
        assert l == "%-20s %3d %s" % (key, idx, val)
        assert entries[key][idx] == val
        parsed.append((key, idx))
    assert parsed[0][0] == "OUTPUTBASE" and parsed[-1][0] == "PRINTTIMER"
    assert len(lines) == sum(len(v) for v in entries.values())
    assert [i for k, i in parsed if k == "FPTCG"] == list(range(7))


@pytest.mark.parametrize("edit,msg", [
    (lambda t: t.replace("X0                   -2.9\n", ""), "(X0) must be specified at least once"),
    (lambda t: t + "X0 1.0\n", "(X0) can be specified only once"),
    (lambda t: t.replace("BARRIERHEIGHTS       7.20 2.00", "BARRIERHEIGHTS 7.2"), "requires exactly 2 values"),
    (lambda t: t + "NOSUCHKEY 1\n", "undefined option (NOSUCHKEY)"),
])
def test_grammar_errors(edit, msg):
    with pytest.raises(ldp.LdpError) as e:
        ldp.params_from_inp_text(edit(quick_text()))
    assert e.value.status == 6
    assert msg in str(e.value)


def test_default_inp_round_trip(tmp_path):
    for model in (ldp.MODEL_SINGLE, ldp.MODEL_DOUBLE):
        path = str(tmp_path / f"d{model}.inp")
        assert L.lib().ldp_write_default_inp(path.encode(), model) == 0
        text = open(path).read()
        assert text.startswith("# [Output] Output base\nOUTPUTBASE           langevinDynamicsSingleBarrier\n")
        p = ldp.params_from_inp(path, model)
        d = ldp.default_params(model)
        assert bytes(p) == bytes(d)


def test_missing_file_is_io_error():
    with pytest.raises(ldp.LdpError) as e:
        ldp.params_from_inp("/nonexistent/x.inp")
    assert e.value.status == 5


def test_no_device_is_reported_not_faked():
    # On a machine without a GPU the context cannot be created; on a GPU
    # machine this just creates and destroys one.
    h = C.c_void_p()
    st = L.lib().ldp_create(C.byref(h), 0)
    if st == 0:
        L.lib().ldp_destroy(h)
    else:
        assert st == 3
