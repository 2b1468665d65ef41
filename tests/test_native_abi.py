"""Host-side checks of the C-ABI library: loads, exports every declared
symbol, rejects bad arguments without a device, and its host BVH builder
reproduces the reference builder bit-for-bit."""
import ctypes
import hashlib
import os
import re

import numpy as np
import pytest

import oracle
from tests.conftest import cuda_available
from tests.golden import cases
from vkpathtracer_b200 import native, scenes

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "vkptc.h")).read()
    return sorted(set(re.findall(r"^\s*(?:int32_t|uint32_t|const char\*)\s+(vkptc_\w+)\s*\(", text, re.M)))


def test_abi_version_matches_the_header():
    """vkptc_abi_version() is the VKPTC_ABI_VERSION the library was built with;
    the bindings refuse a library with another struct layout."""
    text = open(os.path.join(ROOT, "include", "vkptc.h")).read()
    declared = int(re.search(r"#define VKPTC_ABI_VERSION (\d+)u", text).group(1))
    assert native.load().vkptc_abi_version() == declared == native.ABI_VERSION


def test_library_exports_every_declared_symbol():
    lib = native.load()
    syms = declared_symbols()
    assert len(syms) >= 20
    for s in syms:
        assert hasattr(lib, s), s
    assert set(syms) == set(native.SIGNATURES), "ctypes signature table out of sync with include/vkptc.h"


def test_null_arguments_rejected_without_device():
    lib = native.load()
    assert lib.vkptc_configure(None, None) == native.INVALID_ARGUMENT
    assert lib.vkptc_render(None, None, 0, 0, None) == native.INVALID_ARGUMENT
    assert lib.vkptc_create(None, None) == native.INVALID_ARGUMENT
    assert lib.vkptc_last_error(None) == b"null context"


@pytest.mark.skipif(cuda_available(), reason="checks the no-device path")
def test_create_without_device_is_unsupported():
    lib = native.load()
    h = ctypes.c_void_p()
    assert lib.vkptc_create(None, ctypes.byref(h)) == native.UNSUPPORTED
    assert not h.value


def product_binary_bvh(scene):
    lib = native.load()
    v = native.SceneView()
    keep = (scene.vertices, scene.indices, scene.instances)
    v.vertices, v.vertex_count = keep[0].ctypes.data, keep[0].shape[0]
    v.indices, v.index_count = keep[1].ctypes.data, keep[1].size
    v.instances, v.instance_count = keep[2].ctypes.data, keep[2].shape[0]
    n = scene.triangle_count
    nodes = np.zeros((2 * n - 1, 10), np.uint32)
    prim = np.zeros(n, np.uint32)
    nc, pc = ctypes.c_uint32(), ctypes.c_uint32()
    rc = lib.vkptc_build_binary_bvh(ctypes.byref(v), nodes.ctypes.data, ctypes.byref(nc), prim.ctypes.data,
                                    ctypes.byref(pc))
    assert rc == native.OK
    return nodes[: nc.value], prim[: pc.value]


@pytest.mark.parametrize("name", ["box", "field", "sphere"])
def test_product_bvh_builder_matches_reference_golden(name):
    d = cases.load_fixture(name)
    nodes, prim = product_binary_bvh(cases.scene_from_arrays(d))
    h = np.frombuffer(hashlib.sha256(nodes.tobytes() + prim.tobytes()).digest(), np.uint8)
    assert np.array_equal(h, d["bvh_nodes_sha256"])


def test_product_bvh_builder_matches_oracle_on_larger_scene():
    sc = scenes.sphere_field(6, 12, 14, seed=8)
    a_nodes, a_prim = product_binary_bvh(sc)
    b_nodes, b_prim = oracle.load("auto").build_bvh(sc)
    assert np.array_equal(a_nodes, b_nodes)
    assert np.array_equal(a_prim, b_prim)
