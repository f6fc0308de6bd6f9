"""qcstorm_b200: B200-native QC-STORM MLEbfgs localization (Python side).

The product is the C ABI library lib/libqcstorm_b200.so (include/qcstorm_b200.h);
this package holds its ctypes binding and the seeded synthetic-data generators.
"""
from .abi import LocPara, default_para  # noqa: F401
