"""The library's device memory pool.

Runs allocate their buffers from a per-device pool of the library that keeps released blocks for
the next run (h1d_create / h1d_destroy no longer map and unmap device memory each time).  Checked
here: the same run created, stepped and destroyed six times leaves device memory use where the
first cycle left it, and h1d_trim_device_memory gives the pool's unused blocks back to the driver.
"""
import pytest

import hfemic_b200 as h

pytestmark = pytest.mark.gpu
MB = 1 << 20


def _cycle(gpu_lib, cfg, seed):
    with h.Run(cfg, gpu_lib, "h1d_") as r:
        h.abi.populate_state(r, seed)
        r.advance(3)
        r.energy()


@pytest.mark.parametrize("precision", [h.configs.PREC_FP64, h.configs.PREC_MIXED])
def test_repeated_runs_reuse_pooled_memory(gpu_lib, precision):
    import torch

    cfg = h.configs.ensemble_member(3, precision=precision, ppc_scale=0.5)
    held0 = h.abi.trim_device_memory(gpu_lib, 0)  # blocks of any run still alive elsewhere
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    _cycle(gpu_lib, cfg, 0)
    free1 = torch.cuda.mem_get_info()[0]
    held1 = h.abi.trim_device_memory(gpu_lib, 1 << 62)  # keeps everything: only reads the size
    assert held1 > held0, "the released run's blocks stay in the pool"
    for seed in range(1, 6):
        _cycle(gpu_lib, cfg, seed)
    free6 = torch.cuda.mem_get_info()[0]
    held6 = h.abi.trim_device_memory(gpu_lib, 1 << 62)
    assert held6 <= held1 + 16 * MB, (held1, held6)
    assert free6 >= free1 - 16 * MB, (free1, free6)
    # a trim to zero returns every block no run uses
    assert h.abi.trim_device_memory(gpu_lib, 0) <= held0 + 16 * MB
    assert torch.cuda.mem_get_info()[0] >= free0 - 16 * MB
