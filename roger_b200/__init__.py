"""B200-native (sm_100a) JPEG 2000 encode/decode hot path with roger's operator interface.

The compute lives in libj2kb200.so (roger_b200/csrc, C ABI in include/j2k_b200.h).  This
package is the host-side mirror of the reference's classes (OCLEncoder, OCLDecoder,
OCLDWTForward, OCLDWTRev, OCLRGBtoPlanar, OCLBPC) plus the synthetic input generators.
"""
__version__ = "0.1.0"


def __getattr__(name):
    # the torch-backed API is imported lazily so that `import roger_b200` stays cheap
    if name in ("codec", "synth", "diff97", "batch", "shard"):
        import importlib
        return importlib.import_module(f"{__name__}.{name}")
    raise AttributeError(name)
