"""The C++ host engine's plan handling without a GPU: parse errors carry a
line number, node types off the GPU path are refused, and without a device
the driver fails loudly (no CPU fallback)."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "pythia-core_b200", "host", "pyg_executequery")


def run(tmp_path, text):
    p = tmp_path / "plan.conf"
    p.write_text(text)
    return subprocess.run([EXE, str(p)], cwd=tmp_path, capture_output=True, text=True, timeout=60)


def test_parse_error_reports_line(tmp_path):
    r = run(tmp_path, 'path = "./";\nbuffsize = 1024;\nscan: { type = "parallelscan"; files = ( "a" ;\n')
    assert r.returncode == 1 and "line" in r.stderr


def test_unsupported_node_type_is_refused(tmp_path):
    r = run(tmp_path, 'path = "./";\nbuffsize = 1024;\n'
                      'scan: { type = "parallelscan"; filetype = "binary"; files = ("x.bin"); mapping = ((0)); '
                      'schema = ("long"); };\n'
                      'f: { type = "filter"; };\n'
                      'treeroot: { name: "f"; input: { name: "scan"; }; };\n')
    assert r.returncode == 1 and "not on the GPU" in r.stderr


def test_non_integer_column_is_refused(tmp_path):
    r = run(tmp_path, 'path = "./";\nbuffsize = 1024;\n'
                      'scan: { type = "parallelscan"; filetype = "binary"; files = ("x.bin"); mapping = ((0)); '
                      'schema = ("dec"); };\ntreeroot: { name: "scan"; };\n')
    assert r.returncode == 1 and "dec" in r.stderr


def test_no_gpu_fails_loudly(tmp_path):
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    (tmp_path / "x.bin").write_bytes(b"\0" * 16)
    r = run(tmp_path, 'path = "./";\nbuffsize = 1024;\n'
                      'scan: { type = "parallelscan"; filetype = "binary"; files = ("x.bin"); mapping = ((0)); '
                      'schema = ("long", "long"); };\ntreeroot: { name: "scan"; };\n')
    assert r.returncode == 3 and "device" in r.stderr
