"""Host-side checks of the torch.autograd binding (no GPU needed): it refuses tensors that are
not float64 CUDA tensors instead of falling back to any CPU path."""
import pytest

torch = pytest.importorskip("torch")


def test_rejects_host_tensors():
    from axtb_b200.torch_ops import GFN2Energy

    with pytest.raises(TypeError):
        GFN2Energy.apply(torch.zeros((3, 3), dtype=torch.float64), None)


def test_rejects_single_precision():
    from axtb_b200.torch_ops import GFN2Energy

    x = torch.zeros((3, 3), dtype=torch.float32)
    with pytest.raises(TypeError):
        GFN2Energy.apply(x, None)
