"""Sanitizer fuzzing on the CPU (no kernel is launched).  The host tier-2 reader and writer
(t2.cpp), the tier-1 block decoder (t1dec.cu, whose decode_block is the device kernel's own code,
run through its host entry point) and PCRD-opt (rate.cpp) are compiled with AddressSanitizer and
UBSan into the drivers under tests/cpp/, and fed mutated codestreams, random codewords and random
block sets: no out-of-bounds access, no undefined behaviour, every mutant refused with a status
or parsed consistently, every cut within its budget."""
import os
import shutil
import subprocess

import pytest

from oracle import oracle as O
from roger_b200 import synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "roger_b200", "csrc")
LIBDIR = os.path.join(ROOT, "roger_b200")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
SAN = ["-fsanitize=address,undefined", "-fno-sanitize-recover=undefined", "-fno-omit-frame-pointer"]
ENV = dict(os.environ, ASAN_OPTIONS="detect_leaks=0:abort_on_error=0:exitcode=99",
           UBSAN_OPTIONS="print_stacktrace=1:halt_on_error=1:exitcode=98")

pytestmark = pytest.mark.skipif(shutil.which("g++") is None or not os.path.exists(os.path.join(CUDA, "bin", "nvcc")),
                                reason="needs g++ and nvcc")


def _run(cmd, **kw):
    r = subprocess.run(cmd, capture_output=True, text=True, **kw)
    assert r.returncode == 0, (r.returncode, r.stdout[-2000:], r.stderr[-4000:])
    return r.stdout


def _link(tmp_path, name, objs_or_srcs, extra=()):
    from roger_b200 import _lib
    _lib.lib()  # the library provides everything the instrumented unit does not
    exe = str(tmp_path / name)
    _run(["g++", "-std=c++17", "-O1", "-g"] + SAN + ["-I", os.path.join(ROOT, "include"), "-I", CSRC, "-I",
         os.path.join(CUDA, "include")] + list(objs_or_srcs) + ["-o", exe, "-L", LIBDIR, "-lj2kb200",
         "-Wl,-rpath," + LIBDIR, "-L", os.path.join(CUDA, "lib64"), "-lcudart",
         "-Wl,-rpath," + os.path.join(CUDA, "lib64"), "-pthread"] + list(extra))
    return exe


def test_t2_reader_under_sanitizers(tmp_path):
    PIL = pytest.importorskip("PIL.Image")
    import io
    seeds = [bytes(O.encode_image(synth.rgb(96, 80, (5, 6, 7, 8)), 3, 32, 32, True)),
             bytes(O.encode_image(synth.gray(131, 97, 9), 4, 64, 64, True)),
             bytes(O.encode_image(synth.gray(90, 70, 3), 3, 16, 16, True, style=O.STYLE_BYPASS | O.STYLE_TERMALL)),
             bytes(O.encode_image(synth.rgb(64, 64, (1, 2, 3, 4)), 3, 32, 32, False, style=7))]
    buf = io.BytesIO()
    PIL.fromarray(synth.rgb(72, 56, (11, 12, 13, 14))).save(
        buf, "JPEG2000", irreversible=False, mct=1, num_resolutions=4, codeblock_size=(16, 16), progression="RLCP",
        quality_mode="rates", quality_layers=[40, 10, 1], no_jp2=True)
    seeds.append(buf.getvalue())
    paths = []
    for i, cs in enumerate(seeds):
        p = tmp_path / f"seed{i}.j2k"
        p.write_bytes(cs)
        paths.append(str(p))
    exe = _link(tmp_path, "fuzz_t2_reader",
                [os.path.join(ROOT, "tests", "cpp", "fuzz_t2_reader.cpp"), os.path.join(CSRC, "t2.cpp")])
    out = _run([exe, "3000"] + paths, env=ENV, timeout=600)
    parsed, refused, rewritten = int(out.split()[1]), int(out.split()[3]), int(out.split()[7])
    assert parsed > 0 and refused > 0 and rewritten > 0, out


def test_t1_block_decoder_under_sanitizers(tmp_path):
    obj = str(tmp_path / "t1dec_san.o")
    _run([os.path.join(CUDA, "bin", "nvcc"), "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++17", "-O1", "-g",
          "-Xcompiler", "-fsanitize=address,-fsanitize=undefined,-fno-sanitize-recover=undefined,-fno-omit-frame-pointer",
          "-I", os.path.join(ROOT, "include"), "-I", CSRC, "-c",
          os.path.join(CSRC, "t1dec.cu"), "-o", obj])
    exe = _link(tmp_path, "fuzz_t1_block_decode", [os.path.join(ROOT, "tests", "cpp", "fuzz_t1_block_decode.cpp"), obj])
    out = _run([exe, "20000"], env=ENV, timeout=600)
    assert int(out.split()[1]) > 15000, out


def test_pcrd_under_sanitizers(tmp_path):
    """PCRD-opt (rate.cpp) on random block sets, up to 9000 blocks: every cut keeps whole passes
    within the codeword and fits the budget, whatever the plane-end positions and distortions."""
    exe = _link(tmp_path, "fuzz_pcrd", [os.path.join(ROOT, "tests", "cpp", "fuzz_pcrd.cpp"), os.path.join(CSRC, "rate.cpp")])
    out = _run([exe, "200"], env=ENV, timeout=600)
    assert int(out.split()[1]) == 1200, out

