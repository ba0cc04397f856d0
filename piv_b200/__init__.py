"""piv_b200 — B200-native PIV multipass analysis (FFT cross-correlation, sub-pixel peak fit,
normalized-median validation) behind a C ABI, with a Python mirror of the reference's
`piv-core` interface."""
from .api import (  # noqa: F401
    RAW,
    ConfigError,
    CudaError,
    Grid,
    ImageTooSmallError,
    MaskConfig,
    PairResult,
    PassTrace,
    PivBatch,
    PivPipeline,
    PivAnalyzer,
    PivConfig,
    PivError,
    PivServer,
    PreparedFrame,
    PreprocessConfig,
    ShapeMismatchError,
    UnsupportedError,
    ValidationConfig,
    ValidationSummary,
    VectorField,
    flags,
)
from ._lib import LIB_PATH, load as load_library  # noqa: F401
