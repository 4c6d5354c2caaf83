"""ImageStack's .tmp format: round trips, and files exchanged with the reference's own
loader and saver (its CLI built under oracle/_ref)."""
import os
import subprocess

import numpy as np
import pytest

import oracle
from imagestack_b200 import synth
from imagestack_b200.tmpfile import load_tmp, save_tmp

CLI = oracle.REF_CLI


def test_round_trip_every_type(tmp_path):
    # values in [0, 100]: inside every type's range (out-of-range casts have no defined result)
    img = synth.image(37, 21, 3, rects=4, seed=3) * 100.0
    for t in ("float32", "float64", "uint8", "int8", "uint16", "int16", "uint32", "int32",
              "uint64", "int64"):
        p = str(tmp_path / ("a_%s.tmp" % t))
        save_tmp(p, img, t)
        back = load_tmp(p)
        assert back.shape == img.shape and back.dtype == np.float32
        if t.startswith("float"):
            np.testing.assert_array_equal(back, img)
        else:   # the C cast truncates toward zero
            np.testing.assert_array_equal(back, np.trunc(img))


def test_frames_and_bad_files(tmp_path):
    vid = np.arange(2 * 3 * 4 * 5, dtype=np.float32).reshape(2, 3, 4, 5)
    p = str(tmp_path / "v.tmp")
    save_tmp(p, vid)
    np.testing.assert_array_equal(load_tmp(p), vid)
    with open(p, "r+b") as f:
        f.truncate(20 + 4 * 10)
    with pytest.raises(ValueError):
        load_tmp(p)
    with pytest.raises(ValueError):
        save_tmp(p, vid, "float16")


@pytest.mark.skipif(not os.path.exists(CLI), reason="reference CLI not built")
@pytest.mark.parametrize("kind", ["float32", "int16"])
def test_files_exchange_with_the_reference_cli(tmp_path, kind):
    img = synth.image(29, 17, 3, rects=4, seed=5) * 100.0
    ours = str(tmp_path / "ours.tmp")
    theirs = str(tmp_path / "theirs.tmp")
    save_tmp(ours, img)
    # the reference loads our file and saves it in the given type
    subprocess.run([CLI, "-load", ours, "-save", theirs, kind], check=True,
                   capture_output=True, timeout=60)
    mine = str(tmp_path / "mine.tmp")
    save_tmp(mine, img, kind)
    with open(theirs, "rb") as a, open(mine, "rb") as b:
        assert a.read() == b.read()          # byte-identical files
    np.testing.assert_array_equal(load_tmp(theirs), load_tmp(mine))
