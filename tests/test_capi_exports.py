"""The C-ABI library loads on a host without a GPU and exports every
function declared in include/*.h."""
import ctypes
import os
import re

INCLUDE = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include")


def declared_functions():
    names = set()
    for fn in os.listdir(INCLUDE):
        if not fn.endswith(".h"):
            continue
        text = open(os.path.join(INCLUDE, fn)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\(", text):
            name = m.group(1)
            if name in ("if", "defined", "sizeof", "float", "return", "void"):
                continue
            # only declarations at statement level: preceded by a type
            line = text[text.rfind("\n", 0, m.start()) + 1: m.start()]
            if re.search(r"(int|void|double|char\s*\*|const char\s*\*|long long|size_t|\*)\s*$",
                         line.strip() + " ") or line.strip().endswith(("int", "void", "double", "*")):
                names.add(name)
    return names


def test_library_exports_every_declared_symbol():
    from cola_halo_b200 import _lib
    lib = ctypes.CDLL(_lib.lib_path() if os.path.exists(_lib.lib_path()) else _lib.load()._name)
    names = declared_functions()
    assert {"pm_init", "pm_calculate_forces", "cola_kick", "cola_drift", "cola_set_snapshot",
            "lpt_init", "lpt_set_displacement", "lpt_get_local_nx", "power_init", "PowerSpec",
            "GrowthFactor", "move_particles2", "cg_sim_create", "cg_last_error"} <= names
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_exports():
    from cola_halo_b200 import _lib
    names = declared_functions()
    assert names <= set(_lib.SIGNATURES), sorted(names - set(_lib.SIGNATURES))


def test_device_count_without_gpu_is_safe():
    from cola_halo_b200 import _lib
    lib = _lib.load()
    assert lib.cg_device_count() >= 0
    assert lib.cg_mesh_supported(768) == 1 and lib.cg_mesh_supported(770) == 0
