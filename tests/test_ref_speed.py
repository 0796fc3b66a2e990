"""GPU: the reference's own CUDA kernels (compiled from the reference sources
into oracle/_ref, launched with the reference geometry) against this
library's kernels on the same inputs and the same GPU: every (order,
precision) pair must be faster here.  Times are printed (run with -s)."""
import os
import time

import numpy as np
import pytest

import sapporo2_b200 as sp
from oracle import oracle as O
from tests import cases as T

pytestmark = pytest.mark.gpu

# all-i sweep: N^2 interactions per launch (32768: 1.07e9); SAPB_REF_SPEED_N overrides
N = int(os.environ.get("SAPB_REF_SPEED_N", "32768"))


@pytest.mark.parametrize("order,precision", [(1, sp.DOUBLESINGLE), (1, sp.DOUBLE),
                                             (2, sp.DOUBLESINGLE), (2, sp.DOUBLE)])
def test_faster_than_reference_kernels(gpu, order, precision):
    torch = pytest.importorskip("torch")
    if not O.ref_available():
        pytest.skip("oracle/_ref not built")
    case = T.build_case(order, N, seed=71, binaries=0.1)
    rpx, rpv, rpa = O.ref_predict(order, case["ti"], case["t0"], case["x"], case["m"],
                                  case["v"], case["a"], case["j"], case["s"], case["c"])
    pa = rpa if order == 2 else None
    ref = O.ref_gravity(order, precision, rpx, rpv, pa, case["h2"], case["id"], rpx, rpv, pa,
                        case["m"], case["id"], case["eps2"], reps=3)
    n = case["n"]
    with sp.Sapporo(order=order, precision=precision) as s:
        stream = torch.cuda.Stream()
        s.set_stream(stream.cuda_stream)
        s.set_j_particles(np.arange(n), case["id"], case["t0"], case["m"], case["x"], case["v"],
                          case["a"], case["j"], case["s"], case["c"])
        s.set_time(case["ti"])
        s.force_prediction(n)
        rec = sp.pack_i_records(order, rpx, rpv, case["h2"], case["id"], pa)
        i_dev = torch.from_numpy(rec).cuda()
        res = torch.zeros((n, sp.RES_STRIDE), dtype=torch.float64, device="cuda")
        cnt = torch.zeros(n, dtype=torch.int32, device="cuda")
        lst = torch.zeros(n * sp.NGB_PB, dtype=torch.int32, device="cuda")
        times = []
        for it in range(4):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            rc = s.lib.sapb_force_device(s.dev, n, n, i_dev.data_ptr(), case["eps2"],
                                         sp.F_NGB_LIST, res.data_ptr(), cnt.data_ptr(),
                                         lst.data_ptr())
            e1.record(stream)
            assert rc == 0
            e1.synchronize()
            if it:
                times.append(e0.elapsed_time(e1))
        out = res.cpu().numpy()
    mine = float(np.median(times))
    got = {"acc": out[:, 0:3], "pot": out[:, 3], "jrk": out[:, 4:7]}
    T.check_forces(got, ref, order, fields=["acc", "pot", "jrk"])
    inter = float(n) * n
    print(f"\norder {2 * order + 2} prec {'DS' if precision == 1 else 'DP'}: reference "
          f"{ref['ms']:.2f} ms ({inter / ref['ms'] / 1e6:.1f} G int/s), this library "
          f"{mine:.2f} ms ({inter / mine / 1e6:.1f} G int/s), speed-up {ref['ms'] / mine:.2f}x")
    assert mine < ref["ms"]
