"""Plan wisdom: the autotuner's choices saved to and loaded from a text file.

CPU tests cover the file format (header, foreign device types kept, malformed
lines and unknown variants ignored, errors for missing or foreign files).  The
GPU tests show that an imported choice is the one a later plan uses, and that
FFT3D_B200_WISDOM persists a choice from one process to the next.
"""
import os
import subprocess
import sys

import pytest

import fft3d_b200 as fb

HEADER = "fft3d_b200 wisdom 1\n"
FOREIGN = "Some Other GPU|sm9.0|132\t17 17 17 0 -1 11\tstream 17x17x17 double alg0 vpc1 nt320 st2 minb1"


def test_foreign_entries_round_trip(tmp_path):
    fb.wisdom_forget()
    src = tmp_path / "w.txt"
    src.write_text(HEADER + FOREIGN + "\n" + "not a wisdom line\n" + "\n")
    assert fb.wisdom_import(src) == 0  # no device of that type here
    dst = tmp_path / "w2.txt"
    fb.wisdom_export(dst)
    lines = dst.read_text().splitlines()
    assert lines[0] == HEADER.strip()
    assert FOREIGN in lines
    assert "not a wisdom line" not in lines
    # importing the same file twice keeps one copy of the foreign line
    fb.wisdom_import(src)
    fb.wisdom_export(dst)
    assert dst.read_text().splitlines().count(FOREIGN) == 1
    fb.wisdom_forget()


def test_bad_files_are_refused(tmp_path):
    with pytest.raises(fb.Fft3dError):
        fb.wisdom_import(tmp_path / "missing.txt")
    other = tmp_path / "other.txt"
    other.write_text("some other format\n")
    with pytest.raises(fb.Fft3dError):
        fb.wisdom_import(other)
    with pytest.raises(fb.Fft3dError):
        fb.wisdom_export(tmp_path / "no_such_dir" / "w.txt")


def _device_tag(path):
    for line in open(path).read().splitlines()[1:]:
        tag, key, name = line.split("\t")
        if key.startswith("8 8 8 0 -1"):
            return tag
    raise AssertionError("no 8^3 entry was exported")


@pytest.mark.gpu
def test_imported_choice_is_used(tmp_path):
    fb.wisdom_forget()
    shape, b = (8, 8, 8), 100
    fb.Plan(shape, b, fb.FORWARD, fb.C128).close()  # tunes and remembers
    out = tmp_path / "tuned.txt"
    assert fb.wisdom_export(out) >= 1
    tag = _device_tag(out)
    # pin a variant the tuner may not have chosen: the plan must take it untimed
    names = fb.variants(shape, fb.C128, fb.FORWARD)
    pick = names[-1]
    bucket = b.bit_length() - 1
    forced = tmp_path / "forced.txt"
    forced.write_text(HEADER + f"{tag}\t8 8 8 0 -1 {bucket}\t{pick}\n")
    fb.wisdom_forget()
    assert fb.wisdom_import(forced) >= 1
    p = fb.Plan(shape, b, fb.FORWARD, fb.C128)
    assert p.describe() == pick
    p.close()
    fb.wisdom_forget()


@pytest.mark.gpu
def test_environment_variable_persists_across_processes(tmp_path):
    path = tmp_path / "env_wisdom.txt"
    code = ("import sys; sys.path.insert(0, %r); import fft3d_b200 as fb; "
            "p = fb.Plan((12, 12, 12), 64, fb.FORWARD, fb.C128); print(p.describe())"
            % os.path.join(os.path.dirname(__file__), "..", "opt-fft_b200"))
    env = dict(os.environ, FFT3D_B200_WISDOM=str(path))
    first = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True,
                           timeout=300)
    assert first.returncode == 0, first.stderr
    text = path.read_text()
    assert "\t12 12 12 0 -1 6\t" in text
    chosen = [ln.split("\t")[2] for ln in text.splitlines()[1:] if "\t12 12 12 0 -1 6\t" in ln][0]
    assert first.stdout.strip() == chosen
    second = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True,
                            timeout=300)
    assert second.returncode == 0, second.stderr
    assert second.stdout.strip() == chosen
