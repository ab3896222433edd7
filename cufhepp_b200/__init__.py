"""cufhepp_b200: a B200-native TFHE gate-bootstrapping engine with the gate
API of cuFHEpp (Initialize/CleanUp, gates on a Stream, Synchronize).

The engine is the C-ABI library ``lib/libcufhe_b200.so`` (declared in
``include/cufhe_b200.h``); ``cufhepp_b200.gates`` mirrors the reference's
gate API over it, and ``cufhepp_b200.client`` provides key generation,
encryption and decryption.
"""
from . import params  # noqa: F401
