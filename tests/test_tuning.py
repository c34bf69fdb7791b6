"""Launch-shape tuning: the autotuner's table reaches the library
(sb_set_tuning), and -- on the GPU -- every compiled shape keeps parity with
the FP64 oracle, the CTA count leaves results bit-identical, and shapes the
library does not have are refused."""
import numpy as np
import pytest

from specklesource_b200 import abi, autotune


class _Lib:
    def __init__(self):
        self.calls = []

    def sb_set_tuning(self, h, kernel, window, threads, ctas):
        self.calls.append((kernel, window, threads, ctas))
        return abi.SB_OK if window in (16, 24, 32, 48, 64) else abi.SB_ERR_UNSUPPORTED


class _Ctx:
    def __init__(self):
        self.lib = _Lib()
        self.h = None


def test_apply_passes_every_entry_and_skips_refused_ones():
    table = {"entries": [{"kernel": "complex", "window": 64, "threads": 512, "ctas_per_sm": 1},
                         {"kernel": "complex_tc", "window": 64, "threads": 0, "ctas_per_sm": 2},
                         {"kernel": "amplitude", "window": 40, "threads": 0, "ctas_per_sm": 1},
                         {"kernel": "unknown", "window": 32}]}
    c = _Ctx()
    assert autotune.apply(c, table) == 2
    assert c.lib.calls == [(abi.SB_TUNE_COMPLEX, 64, 512, 1), (abi.SB_TUNE_COMPLEX_TC, 64, 0, 2),
                           (abi.SB_TUNE_AMPLITUDE, 40, 0, 1)]


@pytest.mark.gpu
def test_every_compiled_shape_keeps_parity():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from oracle import oracle
    from specklesource_b200 import build, runtime, synth

    from .parity import compare_track
    build.build()
    s1, s2 = synth.small_pair(na=512, nr=1024)
    a, b = synth.to_numpy(s1), synth.to_numpy(s2)
    with runtime.Context(0, tuning=False) as ctx:
        assert ctx.lib.sb_set_tuning(ctx.h, abi.SB_TUNE_COMPLEX, 40, 0, 0) == abi.SB_ERR_UNSUPPORTED
        assert ctx.lib.sb_set_tuning(ctx.h, abi.SB_TUNE_COMPLEX, 64, 96, 0) == abi.SB_ERR_UNSUPPORTED
        assert ctx.lib.sb_set_tuning(ctx.h, abi.SB_TUNE_COMPLEX, 64, 256, 64) == abi.SB_ERR_ARG
        for W, ths in autotune.COMPLEX_THREADS.items():
            p = abi.TrackParams(rStart=W + 8, aStart=W + 8, deltaR=W // 2, deltaA=W // 2, nR=(1024 - 2 * W - 16) // (W // 2),
                                nA=(512 - 2 * W - 16) // (W // 2), wR=W, wA=W, wRa=W, wAa=W)
            o = oracle.strack(p, a, b)
            for t in ths:
                ref = None
                for ctas in (1, 2):
                    if ctx.lib.sb_set_tuning(ctx.h, abi.SB_TUNE_COMPLEX, W, t, ctas) != abi.SB_OK:
                        continue
                    g = ctx.strack(p, a, b)
                    st = compare_track(g, o)
                    assert st["pass"], (W, t, ctas, st)
                    if ref is None:
                        ref = g
                    else:  # the CTA count does not change results
                        for k in ("offR", "offA", "corr", "type"):
                            assert np.array_equal(ref[k], g[k]), (W, t, k)
            ctx.lib.sb_set_tuning(ctx.h, abi.SB_TUNE_COMPLEX, W, 0, 0)
