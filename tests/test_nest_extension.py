"""The NEST extension module (nest-simulator_b200/nest_extension): the
mapping of the C ABI's status codes onto the reference's exceptions, and the
module compiled and linked against the reference's own headers -- the
interface a NEST installation loads (NESTExtensionInterface, Node,
ConnectionManager).  No NEST kernel runs here: the library's NEST symbols
resolve only inside a NEST process."""

import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXT = os.path.join(ROOT, "nest-simulator_b200", "nest_extension")

CODES = {"NG_OK": "none", "NG_ERR_ARG": "BadProperty", "NG_ERR_UNKNOWN_NAME": "BadProperty",
         "NG_ERR_NUMERIC": "NumericalInstability", "NG_ERR_CUDA": "KernelException",
         "NG_ERR_STATE": "KernelException", "NG_ERR_MEMORY": "KernelException",
         "NG_ERR_CAPACITY": "KernelException"}


def test_status_codes_map_to_reference_exceptions(tmp_path):
    src = tmp_path / "map.cpp"
    lines = ['#include <cstdio>', f'#include "{EXT}/ng_errors.h"', "int main() {"]
    for code in CODES:
        lines.append(f'  std::printf("{code} %s\\n", nestgpu::error_kind_name(nestgpu::error_kind({code})));')
    lines += ["  return 0;", "}"]
    src.write_text("\n".join(lines))
    exe = tmp_path / "map"
    subprocess.run(["g++", "-std=c++17", "-o", str(exe), str(src)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = dict(line.split() for line in out if line.strip())
    assert got == CODES


def test_extension_builds_against_reference_headers():
    r = subprocess.run(["make", "-s", "-C", EXT, "check"], capture_output=True, text=True)
    if r.returncode == 2 and "NEST source tree not found" in r.stderr:
        pytest.skip("the reference's source tree is not on this machine")
    assert r.returncode == 0, r.stderr[-3000:]
    so = os.path.join(EXT, "_build", "libnestgpu_module_check.so")
    defined = subprocess.run(["nm", "-D", "--defined-only", so], capture_output=True, text=True).stdout
    names = {line.split()[-1] for line in defined.splitlines() if line.strip()}
    assert {"module", "nestgpu_init"} <= names
    undefined = subprocess.run(["nm", "-DC", "--undefined-only", so], capture_output=True, text=True).stdout
    for sym in ("nest::ModelManager::register_node_model_", "nest::ConnectionManager::get_connections",
                "nest::ConnectionManager::send_to_devices", "nest::ConnectionManager::set_synapse_status",
                "nest::ModelManager::get_connector_defaults", "ng_update", "ng_create",
                "ng_set_plastic_connections", "ng_get_plastic_weights"):
        assert sym in undefined, sym
