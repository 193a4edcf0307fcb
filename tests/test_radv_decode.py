"""CPU tests of the RADV image decoder (rq_radv_describe, host only): its
text equals the reference decoder's (dump_bvh_structure,
include/radv_bvh.hpp:311-390) on the committed golden dumps and, where the
reference library is built, live on images of every shape."""
import ctypes as C
import json
import os

import numpy as np
import pytest

import pyoracle as O
import rq

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_describe_equals_reference_golden_dumps():
    dumps = json.load(open(os.path.join(GOLD, "radv_dumps.json")))
    grids = np.load(os.path.join(GOLD, "ref_dynamic_grids.npz"))
    assert set(dumps) == {"64", "256", "1024", "4096"}
    for n, text in dumps.items():
        img = O.radv_build(grids[f"tri9_{n}"])
        assert rq.radv_describe(img.tobytes()) == text, n


@pytest.mark.skipif(not O.have_ref(), reason="needs oracle/_ref")
@pytest.mark.parametrize("n", [1, 2, 3, 4, 5, 17, 1000, 65537])
def test_describe_equals_live_reference(n):
    tri9 = np.random.default_rng(n).standard_normal(9 * n).astype(np.float32)
    img = O.radv_build(tri9).tobytes()
    assert rq.radv_describe(img) == O.ref_dump_bvh_structure(img)


@pytest.mark.skipif(not O.have_ref(), reason="needs oracle/_ref")
def test_describe_damaged_images_like_reference():
    img = bytearray(O.radv_build(np.random.default_rng(3).standard_normal(9 * 40).astype(np.float32)).tobytes())
    cases = [bytes(img[:100]),                       # shorter than the header
             bytes(img[:200]),                       # root node cut off
             bytes(4096)]                            # all zeros: root at 0, child 0 a "triangle"
    far = bytearray(img)
    far[0:4] = (1 << 20).to_bytes(4, "little")      # bvh_offset past the end
    cases.append(bytes(far))
    odd = bytearray(img)
    odd[192:196] = (0x12345670 | 6).to_bytes(4, "little")  # child 0: an instance far away
    cases.append(bytes(odd))
    for c in cases:
        assert rq.radv_describe(c) == O.ref_dump_bvh_structure(c)


def test_describe_reports_cut_text():
    img = O.radv_build(np.random.default_rng(4).standard_normal(90).astype(np.float32))
    full = rq.radv_describe(img.tobytes())
    buf = C.create_string_buffer(100)
    n = C.c_uint64()
    rc = rq.lib().rq_radv_describe(img.ctypes.data_as(C.c_void_p), img.nbytes, buf, 100, C.byref(n))
    assert rc == rq.RQ_ERR_SIZE and n.value == len(full) and buf.value.decode() == full[:99]
