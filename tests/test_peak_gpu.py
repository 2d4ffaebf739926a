"""The measured FP32 peak (grav_fp32_peak_CUDA), the roofline denominator:
scalar and paired FMA chains, the larger rate, below the nominal FP32 rate
of the device and near it."""
import pytest

pytestmark = pytest.mark.gpu


def test_fp32_peak_near_nominal():
    import torch
    from pgrav import gravcuda as gc
    peak = gc.fp32_peak()
    prop = torch.cuda.get_device_properties(0)
    clock_ghz = 1.965 if prop.major == 10 else 2.0   # B200 maximum SM clock
    nominal = prop.multi_processor_count * 128 * 2 * clock_ghz * 1e9 / 1e12
    assert 0.6 * nominal < peak < 1.03 * nominal, (peak, nominal)
