"""Byte contract: every struct of include/ae_b200.h has the reference's size
and field offsets (scene/gpu_types.h:96-112, scene/bvh.h:43,
scene/mesh_library.h:46, renderer/renderer.h:151-159)."""
import os
import re

from aviatorengine2_b200 import _lib

HDR = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "ae_b200.h")


def test_sizes():
    assert _lib.OBJECT.itemsize == 128
    assert _lib.INSTANCE.itemsize == 48
    assert _lib.NODE.itemsize == 48
    assert _lib.VERTEX.itemsize == 32
    assert _lib.CONFIG.itemsize == 240


def test_object_offsets():
    off = {k: v[1] for k, v in _lib.OBJECT.fields.items()}
    assert off["radius"] == 28 and off["rotation"] == 76 and off["density"] == 80
    assert off["emission"] == 84 and off["textureTint"] == 92 and off["r"] == 96
    assert off["fuzz"] == 108 and off["textureID"] == 124


def test_config_offsets():
    off = {k: v[1] for k, v in _lib.CONFIG.fields.items()}
    assert off["exposure"] == 124 and off["debugView"] == 128 and off["jitter_y"] == 144
    assert off["displayOnly"] == 148 and off["traceScale"] == 152 and off["frameIndex"] == 156
    assert off["historyCap"] == 168 and off["prevViewProj"] == 176


def test_instance_offsets():
    off = {k: v[1] for k, v in _lib.INSTANCE.fields.items()}
    assert off["scale"] == 12 and off["qx"] == 16 and off["vertexBase"] == 32 and off["blasBase"] == 44


def test_header_static_asserts_present():
    src = open(HDR).read()
    assert len(re.findall(r"static_assert\(sizeof\(ae_object\) == 128", src)) == 1
    assert "offsetof(ae_config, prevViewProj) == 176" in src
