"""Host-side device checks of the Python wrappers, without a GPU: a tensor on
another device or in host memory is rejected with ValueError before a pointer
can reach the C ABI (the kernels run on the plan's device; another GPU's
pointer faults it without peer access)."""
import pytest


class FakeTensor:
    def __init__(self, dev):
        self.dev = dev

    def get_device(self):
        return self.dev


def test_require_device():
    from apollofft_b200.plan import require_device
    require_device(FakeTensor(0), 0, "input")
    require_device(FakeTensor(3), 3, "input")
    with pytest.raises(ValueError, match="host memory; the plan is on cuda:0"):
        require_device(FakeTensor(-1), 0, "input")
    with pytest.raises(ValueError, match="output is in cuda:1; the plan is on cuda:0"):
        require_device(FakeTensor(1), 0, "output")
