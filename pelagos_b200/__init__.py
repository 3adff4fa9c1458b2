"""B200-native Relay-BP-S decoder (drop-in for pelagos.RelayBPDecoder).

The decode path is one persistent sm_100a CUDA kernel (csrc/relaybp.cu)
behind the C ABI of include/relaybp.h; this package holds the host side:
argument handling, graph preparation, seeded gamma tables and result
assembly, mirroring the reference's Python interface.
"""

from .adapter import DecodeResult, ObservableDecoderRunner, RelayDecoder, RelayDecoderF32, RelayDecoderF64
from .decoder import RelayBPDecoder, UNCONVERGED_CORRECTIONS

__all__ = ["RelayBPDecoder", "UNCONVERGED_CORRECTIONS", "RelayDecoder", "RelayDecoderF32", "RelayDecoderF64",
           "ObservableDecoderRunner", "DecodeResult"]
__version__ = "0.1.0"
