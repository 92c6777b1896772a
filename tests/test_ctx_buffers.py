"""Every device buffer a context owns is released by lsmps_ctx_destroy: the release list in
ls-mps_b200/csrc/capi.cu names each DevBuf member declared in ls-mps_b200/csrc/ctx.cuh (a
buffer missing there leaks its device memory once per context)."""
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_every_context_buffer_is_released():
    ctx = open(os.path.join(ROOT, "ls-mps_b200", "csrc", "ctx.cuh")).read()
    declared = {n.strip() for m in re.finditer(r"lsmps_gpu::DevBuf\s+([^;]+);", ctx) for n in m.group(1).split(",")}
    capi = open(os.path.join(ROOT, "ls-mps_b200", "csrc", "capi.cu")).read()
    i = capi.index("lsmps_gpu::DevBuf* bufs[]")
    released = set(re.findall(r"&ctx->(\w+)", capi[i:capi.index("};", i)]))
    assert declared and declared <= released, sorted(declared - released)
