"""The C-ABI library loads without a GPU and exports every declared symbol."""
import ctypes
import re
from pathlib import Path

import numpy as np

from rlmusclev2_b200 import _capi as capi
from rlmusclev2_b200.build import build, lib_path

HEADERS = sorted((Path(__file__).resolve().parents[1] / "include").glob("*.h"))


def _declared():
    names = set()
    for h in HEADERS:
        txt = h.read_text()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        names |= set(re.findall(r"^\s*(?:int|const char\*|int32_t|float)\s+(xpbd_\w+)\s*\(", txt, flags=re.M))
    return names


def test_library_loads_and_exports_declared_symbols():
    build()
    lib = ctypes.CDLL(str(lib_path()))
    declared = _declared()
    assert "xpbd_project" in declared and "xpbd_vertex_step" in declared
    for name in declared:
        assert hasattr(lib, name), name
    assert set(capi.exported_symbols()) <= declared | set()
    assert lib.xpbd_abi_version() == 2


def test_struct_sizes_match_header_layout():
    assert ctypes.sizeof(capi.XpbdMaterial) == 32
    assert ctypes.sizeof(capi.XpbdParams) == 64 + 32 * capi.MAX_MATERIALS + 8 * capi.MAX_ATTACH_MATERIALS
    assert ctypes.sizeof(capi.XpbdMetrics) == 32


def test_ctypes_offsets_match_c_compiler(tmp_path):
    """Every ctypes mirror has the field offsets gcc computes from the header."""
    import subprocess
    structs = [capi.XpbdMaterial, capi.XpbdAttachMaterial, capi.XpbdParams, capi.XpbdVerts, capi.XpbdTiles,
               capi.XpbdSdf, capi.XpbdMetrics, capi.XpbdCage, capi.XpbdDcd, capi.XpbdDcdWorkspaceSizes,
               capi.XpbdCapsule, capi.XpbdPersist, capi.XpbdSdfBatch, capi.XpbdGemm, capi.XpbdCageFeatures]
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "xpbd_b200.h"', 'int main(void){']
    for s in structs:
        lines.append(f'printf("{s.__name__} %zu\\n", sizeof({s.__name__}));')
        for f, _ in s._fields_:
            lines.append(f'printf("{s.__name__}.{f} %zu\\n", offsetof({s.__name__}, {f}));')
    lines.append("return 0;}")
    src = tmp_path / "abi.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "abi"
    subprocess.run(["gcc", "-I", str(HEADERS[0].parent), str(src), "-o", str(exe)], check=True)
    out = dict(l.rsplit(" ", 1) for l in subprocess.run([str(exe)], capture_output=True, text=True,
                                                         check=True).stdout.splitlines())
    for s in structs:
        assert int(out[s.__name__]) == ctypes.sizeof(s), s.__name__
        for f, _ in s._fields_:
            assert int(out[f"{s.__name__}.{f}"]) == getattr(s, f).offset, (s.__name__, f)


def test_acc_scale_for_extent_is_the_largest_safe_power_of_two():
    lib = capi.load(build_if_missing=True)
    for e in (1e-4, 0.0137, 0.5, 1.0, 3.17, 100.0, 2500.0):
        s = float(lib.xpbd_acc_scale_for_extent(e))
        k = np.log2(s)
        assert k == round(k)
        assert e * s <= 2.0 ** 26 < e * 2.0 * s
        # quantum at most half an FP32 ulp of the largest coordinate
        assert 1.0 / s <= np.spacing(np.float32(e)) / 2


def test_engine_accumulator_range_rule():
    """The engine sizes the fixed-point range by the larger of 128 longest rest
    edges and the largest rest coordinate: the box muscle's measured worst tet
    correction (97 mm summed over its 12 components) stays inside the range,
    and the 535k-tet scene gets a quantum of at most 3e-8 m."""
    from rlmusclev2_b200.engine import ACC_RANGE_EDGES, max_rest_edge
    from rlmusclev2_b200.meshgen import box_muscle
    lib = capi.load(build_if_missing=True)
    x = np.array([[0, 0, 0], [1, 0, 0], [0, 2, 0], [0, 0, 3]], np.float32)
    assert abs(max_rest_edge(x, np.array([[0, 1, 2, 3]])) - np.sqrt(13.0)) < 1e-6
    m = box_muscle()
    e = max(ACC_RANGE_EDGES * max_rest_edge(m.verts, m.tets), float(np.abs(m.verts).max()))
    s = float(lib.xpbd_acc_scale_for_extent(e))
    assert 2.0 ** 25 / s >= 0.097
    # the 535k-tet scene: longest edge 9.7 mm, largest coordinate 0.96 m
    s2 = float(lib.xpbd_acc_scale_for_extent(max(ACC_RANGE_EDGES * 0.00966, 0.958)))
    assert 1.0 / s2 <= 3e-8 and 2.0 ** 25 / s2 >= 0.25
