"""The allocation-free RADV build (rq_build_radv_noalloc).

It serves callers that own all of their device memory and cannot let a
library call cudaMalloc/cudaFree behind their back (those calls synchronise
the device and can fail under a fixed budget).  Its scratch is a static
device array of bounded size inside librq.so, shared by every call.

This file is collected last on purpose: if the entry point misbehaves, a run
that stops at the first failure has already run every other test.  Each test
works in a fresh process as well as after the rest of the suite."""
import ctypes as C

import numpy as np
import pytest
import torch

import rq
from conftest import soup

pytestmark = pytest.mark.gpu


def noalloc_build(tri9, image):
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    return rq.lib().rq_build_radv_noalloc(C.c_void_p(tri9.data_ptr()), tri9.numel() // 9,
                                          C.c_void_p(image.data_ptr()), image.numel(), stream)


def compare_with_allocating_build(ctx, n, seed):
    tri9 = torch.from_numpy(soup(n, seed).reshape(-1)).cuda()
    want = rq.build_radv(ctx, tri9)
    got = torch.full((rq.radv_size(n),), 0xAB, dtype=torch.uint8, device="cuda")
    assert noalloc_build(tri9, got) == rq.RQ_OK
    torch.cuda.synchronize()
    assert torch.equal(got, want), f"n={n}: allocation-free image differs"


def test_noalloc_matches_allocating_build_twice(ctx):
    # calls in a row, different sizes: the shared scratch keeps the previous
    # call's contents and the result must not depend on them
    for n, seed in ((1 << 20, 91), (5000, 92), (4500000, 93)):
        compare_with_allocating_build(ctx, n, seed)


def test_noalloc_one_block_images(ctx):
    # up to 256 triangles the build is one block and takes no ticket
    for n, seed in ((1, 81), (100, 82), (256, 83), (257, 84), (1, 85)):
        compare_with_allocating_build(ctx, n, seed)


def test_noalloc_at_its_largest_block_counts(ctx):
    # the scratch is sized for the most blocks a build up to the maximum can
    # take: 4,096 blocks at 4,194,300 triangles (256-leaf-box subtrees) and
    # at 2^24 triangles (1,024-leaf-box subtrees)
    for n, seed in ((4194300, 71), (rq.RADV_NOALLOC_MAX_TRIANGLES, 72)):
        compare_with_allocating_build(ctx, n, seed)
        torch.cuda.empty_cache()


def test_noalloc_rejects_misaligned_buffers():
    tri9 = torch.zeros(64, dtype=torch.float32, device="cuda")
    img = torch.zeros(1024, dtype=torch.uint8, device="cuda")
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = rq.lib().rq_build_radv_noalloc(C.c_void_p(tri9.data_ptr() + 2), 1, C.c_void_p(img.data_ptr()), 1024, stream)
    assert rc == rq.RQ_ERR_INVALID_ARG
    rc = rq.lib().rq_build_radv_noalloc(C.c_void_p(tri9.data_ptr()), 1, C.c_void_p(img.data_ptr() + 8), 1000, stream)
    assert rc == rq.RQ_ERR_INVALID_ARG


def test_noalloc_rejects_sizes_beyond_its_scratch():
    tri9 = torch.zeros(9, dtype=torch.float32, device="cuda")
    img = torch.zeros(512, dtype=torch.uint8, device="cuda")
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = rq.lib().rq_build_radv_noalloc(C.c_void_p(tri9.data_ptr()), rq.RADV_NOALLOC_MAX_TRIANGLES + 1,
                                        C.c_void_p(img.data_ptr()), 1 << 40, stream)
    assert rc == rq.RQ_ERR_UNSUPPORTED
    # an image buffer smaller than the layout needs is refused as well
    rc = rq.lib().rq_build_radv_noalloc(C.c_void_p(tri9.data_ptr()), 1, C.c_void_p(img.data_ptr()), 100, stream)
    assert rc == rq.RQ_ERR_SIZE
