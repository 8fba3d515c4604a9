"""B200-native GFN2-xTB energy + analytic gradient (the single point of axtb's calculator).

``Calculator`` and ``Batch`` (axtb_b200.calculator) drive the sm_100a engine in
``libaxtb_gpu.so`` through its C ABI (include/axtb_gpu.h); ``structures`` builds the synthetic
workloads; ``torch_ops`` exposes the batched energy to PyTorch; ``hessian`` gives the
semi-numerical Hessian from one batch of displaced gradients; ``sharding`` spreads molecules
over GPUs.
"""
from .calculator import AxtbError, Batch, Calculator, Moments, SinglePoint, basis_size  # noqa: F401
from .hessian import Hessian, numerical_hessian  # noqa: F401
