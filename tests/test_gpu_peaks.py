"""pmp_measure_peaks: the measured FP64 / FP32 FMA and SFU rates that the
bench's compute roofline divides by.  On a B200 they must sit near the
nominal rates at the clocks the GPU runs (148 SMs x 64 FP64 / 128 FP32 FMA
lanes / 16 SFU lanes per clock, about 1.9 GHz): between a third of nominal
(a throttled or shared GPU) and 10 % above it."""
import pytest

from pelemp_b200.spray import measure_peaks

pytestmark = pytest.mark.gpu


def test_measured_peaks_are_plausible():
    import torch
    p = measure_peaks(torch.cuda.current_device())
    print("measured peaks:", p)
    props = torch.cuda.get_device_properties(torch.cuda.current_device())
    sms = props.multi_processor_count
    ghz = 1.965
    nominal = {"fp64_tflops": sms * 64 * 2 * ghz * 1e-3, "fp32_tflops": sms * 128 * 2 * ghz * 1e-3,
               "sfu_gops": sms * 16 * ghz}
    for k, v in nominal.items():
        assert v / 3 < p[k] < 1.1 * v, (k, p[k], v)
