"""php_fdtd_b200 -- B200 implementation of the PhP_FDTD time-step loop.

Native parts (built in-tree by ``php_fdtd_b200.build``):
  libphpfdtd.so  the CUDA path behind the C ABI of include/php_fdtd.h
  libphphost.so  .cfg / material / medium / output-file layer (C)
  fdtd_b200      drop-in solver executable
"""
from .solver import Config, DescHolder, Material, PhpError, Simulation, Source, make_desc, with_precision  # noqa: F401
from ._abi import COMPONENTS, PREC  # noqa: F401
