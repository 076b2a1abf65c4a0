"""The benchmark's two arms decode the same inputs.

bench.py's GPU arm builds its LLRs with the decoder library (make_data); its CPU
reference arm builds them with the oracle (oracle_data) so that the reference
process never loads the library.  Both must give the same bytes, or the two arms'
numbers would not be on the same workload."""
import numpy as np

import bench


def test_reference_arm_inputs_equal_gpu_arm_inputs():
    for rank in (0, 1):
        info_l, llr_l = bench.make_data(48, rank)
        info_o, llr_o = bench.oracle_data(48, rank)
        assert np.array_equal(info_l, info_o)
        assert llr_l.shape == llr_o.shape == (48, bench.N_TX)
        assert np.array_equal(llr_l, llr_o)


def test_cpu_pipeline_matches_oracle_on_the_workload():
    """The CPU baseline the reference arm times decodes these inputs exactly as the
    oracle does (iterations and packed information bits)."""
    import _oracle as O

    _, llr = bench.oracle_data(24, 0)
    _, its, packed = bench.time_cpu(llr, 24, 3)
    code = O.Code.nr(bench.BG, bench.Z)
    ref = O.decode_i8_batch(code, llr, O.beta_q(bench.BETA), bench.ITERS, llr_offset=bench.PUNCT, nr_prologue=True,
                            hard_bits=bench.K_INFO)
    assert np.array_equal(its, ref["iters"])
    assert np.array_equal(packed, ref["packed"])
