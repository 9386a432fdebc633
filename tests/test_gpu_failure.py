"""Failure paths on the GPU, none of which faults or hangs the device.

The reference stops the process on any CUDA error (src/kc.cu:14-23).  Here
every device-side wait (the grid barriers of the cooperative kernels) has a
bound, the option timeout_ms; when a wait runs past it the kernel sets an
error bit and returns, the call returns KT_ERR_TIMEOUT, and the context stays
usable.  timeout_ms = 0 makes every bounded wait give up at once, which is how
these tests make a wait run out: no kernel is broken and nothing waits
forever."""
import numpy as np
import pytest

import kt_oracle as O
import kc_cuda_b200 as K
from kc_cuda_b200 import gen

pytestmark = pytest.mark.gpu

KT_ERR_INVALID = 1
KT_ERR_TIMEOUT = 6


def test_bounded_wait_gives_up_then_context_recovers():
    g = gen.Graph(gen.rmat(12, 8, 7, [16]))
    data = g.tsv_bytes()
    want = O.solve_tsv(data)
    with K.Context(0) as ctx:
        assert ctx.get_option("persistent") == 1  # cooperative k-core and peel launches
        for _ in range(2):  # twice: the device words must be clean after each failure
            ctx.set_option("timeout_ms", 0)
            with pytest.raises(K.KtError) as ei:
                ctx.solve_tsv(data)
            assert ei.value.status == KT_ERR_TIMEOUT, ei.value
            assert "bounded device wait" in ei.value.message
            ctx.set_option("timeout_ms", 20000)
            assert ctx.solve_tsv(data) == want
        # Stage outputs on a loaded graph recover too.
        dg = ctx.load_tsv(data)
        ctx.set_option("timeout_ms", 0)
        with pytest.raises(K.KtError) as ei:
            dg.core_numbers()
        assert ei.value.status == KT_ERR_TIMEOUT
        ctx.set_option("timeout_ms", 20000)
        assert np.array_equal(dg.core_numbers(), O.core_numbers(g.edges(), g.num_vertices))
        assert dg.kmax_truss() == want
        dg.free()


def test_batch_wait_gives_up_then_batch_runs():
    with K.Context(0) as ctx:
        graphs = [gen.Graph(gen.rmat(9 + i % 3, 8, 100 + i, [10 + i])) for i in range(6)]
        want = [O.solve_tsv(g.tsv_bytes()) for g in graphs]
        for timeout, ok in ((0, False), (20000, True)):
            ctx.set_option("timeout_ms", timeout)
            b = ctx.batch()
            for g in graphs:
                b.add_edges(g.edge_pairs())
            if ok:
                b.run()
                k, c = b.results()
                assert [(int(a), int(e)) for a, e in zip(k, c)] == want
            else:
                with pytest.raises(K.KtError) as ei:
                    b.run()
                assert ei.value.status == KT_ERR_TIMEOUT
            b.free()


def test_option_values_out_of_range(tmp_path):
    with K.Context(0) as ctx:
        for name, v in (("timeout_ms", -1), ("timeout_ms", 3_600_001), ("kcore_window", -5), ("peel_split", -1)):
            before = ctx.get_option(name)
            with pytest.raises(K.KtError) as ei:
                ctx.set_option(name, v)
            assert ei.value.status == KT_ERR_INVALID
            assert ctx.get_option(name) == before
        ctx.set_option("timeout_ms", 3_600_000)
        ctx.set_option("timeout_ms", 20000)
        p = tmp_path / "opts.txt"
        p.write_text("kcore_window -3\n")
        with pytest.raises(K.KtError) as ei:
            ctx.load_options(str(p))
        assert ei.value.status == KT_ERR_INVALID
        assert ctx.get_option("kcore_window") >= 0
