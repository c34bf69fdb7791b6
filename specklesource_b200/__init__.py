"""B200-native (sm_100a) re-implementation of GrIMP speckleSource's hot path:
strack (complex/amplitude speckle tracking), strackw (fast-flow normalised
correlation) and cullst (offset culling), behind the C ABI declared in
include/speckle_b200.h."""
from . import abi  # noqa: F401

__all__ = ["abi"]
