"""B200-native QC-LDPC layered offset min-sum decoder.

Drop-in for syndrome's QC-LDPC decode path (src/qc_ldpc.rs): the same decoder API
in Python (qc_ldpc.py) and C (include/syndrome_ldpc.h), executed by hand-written
sm_100a CUDA kernels (csrc/ldpc_kernels.cu).  There is no CPU decode path: the
decode entry points raise if the CUDA library is not built or no GPU is present.
"""
from ._lib import SyndromeError, load as load_library  # noqa: F401
from .qc_ldpc import (  # noqa: F401
    APP_CLAMP_I8,
    APP_CLAMP_WIDE,
    DEFAULT_SCALE,
    MSG_MAX,
    AwgnChannel,
    BaseGraph,
    BatchResult,
    FecError,
    LdpcWorkspace,
    QcLdpcDecoder,
    QcLdpcEncoder,
    QuantParams,
    awgn_quantized_batch,
    quantize_llr_i16,
    wifi_ldpc_decoder,
    wifi_ldpc_encoder,
)

from .mixed import CODEWORD_DTYPE, LIFTING_SIZES, MixedBatch, code_dims, tile_capacity  # noqa: F401,E402
from .mixed import WIFI_CODEWORD_DTYPE, WIFI_SHAPES, WifiMixedBatch, wifi_dims  # noqa: F401,E402

__version__ = "0.1.0"
from .dlsch import DecodeReport, DlSchDecoder, DlSchEncoder, SegmentationParams, compute_segmentation, crc24  # noqa: F401,E402
from .serve import Server  # noqa: F401,E402
from . import wifi_rate_matching  # noqa: F401,E402
from .ldpc_pipeline import LdpcFrame, LdpcPipeline  # noqa: F401,E402
