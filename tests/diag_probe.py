"""Per-sample radiance from the diagnostic build of libx2 (libx2diag.so, include/x2_diag.h), run as its own process
because the x2 module loads one library a process. Test infrastructure for the parity investigation
(tests/test_gpu_parity_cause.py).

    python tests/diag_probe.py <scene id> <in.npz: pixels, indices> <out.npz> <mode> [library]

mode 0: every sample as the library computes it (no diagnostic switch; any build).
mode 1: every sample with the transcendental functions in double rounded to float -> rgba, status.
mode 2: every sample alone, with CUDA's functions (as the product) and every call recorded -> rgba, status, and the
        records (calls: n x 5 float32 words as x2_diag_call, first: each sample's first record, count: its records).
"""
import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(ROOT, "xpu2-foundation_b200"))
# The library: the diagnostic build, or the one a sixth argument names (e.g. libx2fmad.so, the contracted build).
LIB = sys.argv[5] if len(sys.argv) > 5 else "libx2diag.so"
os.environ["X2_LIBRARY"] = os.path.join(ROOT, "xpu2-foundation_b200", "x2", LIB)

import x2  # noqa: E402

CALL_DTYPE = np.dtype([("fn", np.uint32), ("a", np.float32), ("b", np.float32), ("r0", np.float32), ("r1", np.float32)])


def main(scene_id, src, dst, mode):
    import torch

    lib = x2.library()
    if mode == 0:
        return plain(scene_id, src, dst)
    lib.x2_diag_set.argtypes = [C.c_int, C.c_void_p, C.c_uint32]
    lib.x2_diag_set.restype = C.c_int
    lib.x2_diag_count.argtypes = [C.POINTER(C.c_uint32)]
    lib.x2_diag_count.restype = C.c_int
    f = np.load(src)
    pixels, indices = f["pixels"].astype(np.uint32), f["indices"].astype(np.uint32)
    ctx = x2.Context(0)
    s = x2.SyntheticScene(scene_id)
    scene = x2.Scene(ctx, s.desc, s.config)
    out = {}
    if mode == 1:
        assert lib.x2_diag_set(1, None, 0) == 0
        out["rgba"], out["status"] = scene.integrate(pixels, indices)
    else:
        cap = 1 << 16
        buf = torch.zeros(cap * CALL_DTYPE.itemsize // 4, dtype=torch.int32, device="cuda:0")
        rgba = np.zeros((len(pixels), 4))
        status = np.zeros(len(pixels), np.uint32)
        calls, first, count = [], [], []
        n = C.c_uint32()
        for i in range(len(pixels)):
            assert lib.x2_diag_set(2, C.c_void_p(buf.data_ptr()), cap) == 0
            r, st = scene.integrate(pixels[i:i + 1], indices[i:i + 1])
            rgba[i], status[i] = r[0], st[0]
            assert lib.x2_diag_count(C.byref(n)) == 0 and n.value <= cap
            rec = buf[: n.value * CALL_DTYPE.itemsize // 4].cpu().numpy().view(CALL_DTYPE)
            first.append(sum(len(c) for c in calls))
            count.append(n.value)
            calls.append(rec.copy())
        assert lib.x2_diag_set(0, None, 0) == 0
        out.update(rgba=rgba, status=status, calls=np.concatenate(calls) if calls else np.zeros(0, CALL_DTYPE),
                   first=np.array(first, np.int64), count=np.array(count, np.int64))
    np.savez(dst, pixels=pixels, indices=indices, **out)
    scene.free()
    s.free()
    ctx.close()


def plain(scene_id, src, dst):
    f = np.load(src)
    pixels, indices = f["pixels"].astype(np.uint32), f["indices"].astype(np.uint32)
    ctx = x2.Context(0)
    s = x2.SyntheticScene(scene_id)
    scene = x2.Scene(ctx, s.desc, s.config)
    rgba, status = scene.integrate(pixels, indices)
    np.savez(dst, pixels=pixels, indices=indices, rgba=rgba, status=status)
    scene.free()
    s.free()
    ctx.close()


if __name__ == "__main__":
    main(int(sys.argv[1]), sys.argv[2], sys.argv[3], int(sys.argv[4]))
