"""Regenerates tests/golden/golden.json (run from the repository root: python tests/golden/make_golden.py).

Every codestream fixture is produced by the CPU oracle and, at generation time, decoded by an
independent decoder (OpenJPEG 2.5 inside Pillow, used as a black box): lossless cases must
reconstruct the input exactly, lossy cases record their PSNR.  The tier-1 vectors are single
code-blocks (coefficients -> codeword bytes, symbol count, bit-planes) cut from the 512x512
lossless case.
"""
import hashlib
import io
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from roger_b200 import synth  # noqa: E402

CASES = [
    # name, kind, w, h, seed(s), levels, cb, lossless, embed
    ("gray64_l3_lossless", "gray", 64, 64, 0, 3, 64, True, True),
    ("rgb33x17_l2_cb32_lossless", "rgb", 33, 17, (5, 6, 7, 8), 2, 32, True, True),
    ("gray64x48_l3_cb32_lossy", "gray", 64, 48, 1, 3, 32, False, True),
    ("rgb40x24_l2_lossy", "rgb", 40, 24, (9, 10, 11, 12), 2, 32, False, True),
    ("config0_gray512_l5_lossless", "gray", 512, 512, 0, 5, 64, True, False),
    ("rgb256_l5_cb32_lossless", "rgb", 256, 256, (100, 101, 102, 103), 5, 32, True, False),
]


def image(kind, w, h, seed):
    return synth.gray(w, h, seed) if kind == "gray" else synth.rgb(w, h, seed)


def sha(b):
    return hashlib.sha256(bytes(b)).hexdigest()


def psnr(a, b):
    d = a.astype(np.float64) - b.astype(np.float64)
    m = (d * d).mean()
    return 99.0 if m == 0 else float(10 * np.log10(255.0 ** 2 / m))


def main():
    from PIL import Image
    out = {"generator": "oracle/j2k_oracle.c + roger_b200/synth.py; verified with Pillow "
                        + __import__("PIL").__version__, "codestreams": [], "t1": []}
    for name, kind, w, h, seed, lv, cb, lossless, embed in CASES:
        img = image(kind, w, h, seed)
        cs = O.encode_image(img, lv, cb, cb, lossless)
        dec = np.array(Image.open(io.BytesIO(cs))).reshape(img.shape)
        rec = dict(name=name, kind=kind, w=w, h=h, seed=seed, levels=lv, cb=cb, lossless=lossless,
                   image_sha256=sha(img.tobytes()), codestream_sha256=sha(cs), length=len(cs),
                   openjpeg_exact=bool(np.array_equal(dec, img)), openjpeg_psnr=psnr(dec, img))
        if embed:
            rec["codestream_hex"] = cs.hex()
        if lossless:
            assert rec["openjpeg_exact"], name
        out["codestreams"].append(rec)
    # tier-1 vectors from the config-0 image
    img = synth.gray(512, 512, 0)
    planes = O.planar_fwd(img, O.MCT_NONE)
    coef = O.dwt53_fwd(planes[0], 5)
    for (x0, y0, cw, ch, orient, tag) in [(0, 0, 16, 16, O.LL, "LL5"), (256, 0, 64, 64, O.HL, "HL1"),
                                          (0, 256, 64, 64, O.LH, "LH1"), (256, 256, 64, 64, O.HH, "HH1"),
                                          (128, 128, 64, 64, O.HH, "HH2"), (16, 0, 16, 16, O.HL, "HL5")]:
        blk = np.ascontiguousarray(coef[y0:y0 + ch, x0:x0 + cw])
        data, info, syms = O.t1_encode(blk, orient, want_symbols=True)
        out["t1"].append(dict(tag=tag, x0=x0, y0=y0, cw=cw, ch=ch, orient=orient,
                              coeff=blk.astype(int).flatten().tolist(), codeword_hex=data.hex(),
                              symbols_sha256=sha(syms.tobytes()), **info))
    path = os.path.join(ROOT, "tests", "golden", "golden.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
