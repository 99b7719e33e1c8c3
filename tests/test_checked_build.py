"""The bounds-checked build (libsbfs_checked.so, -DSBFS_CHECKED): every index
the kernels derive from data is checked on the device, and a failed check is
reported as an error status instead of an out-of-bounds access.  The small-n,
hash-set, CTA-wide and golden-fixture parity tests run once against it, in a
child process that loads that library (SBFS_LIB), and must pass unchanged:
no check fires on valid inputs, and the checks do not change any result."""
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CHECKED = os.path.join(ROOT, "gpgpu-binary-automaton-synchronizing-algorithms_b200", "sbfs", "_lib",
                       "libsbfs_checked.so")
SELECTED = " or ".join([
    "test_config1_plain_n8", "test_golden_fixtures_on_every_small_path", "test_uniform_random_each_class",
    "test_n13_16_hash_set_and_pooled_paths", "test_n17_20_hash_set_path_and_hand_offs",
    "test_one_state_automata_match_the_oracle", "test_permutation_automata_on_every_class",
    "test_cerny_known_answers", "test_reference_worst_case_letters", "test_malformed_automaton_is_rejected",
])


def test_parity_under_the_checked_build():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    assert os.path.exists(CHECKED), "build with __graft_entry__.build() first"
    env = dict(os.environ, SBFS_LIB=CHECKED)
    probe = subprocess.run([sys.executable, "-c",
                            "import sys; sys.path.insert(0, sys.argv[1]); import sbfs; sbfs.load(); "
                            "print(sbfs.LIB_PATH); print(any('libsbfs_checked.so' in l for l in open('/proc/self/maps')))",
                            os.path.join(ROOT, "gpgpu-binary-automaton-synchronizing-algorithms_b200")],
                           env=env, capture_output=True, text=True, timeout=120)
    assert probe.returncode == 0, probe.stderr[-2000:]
    assert probe.stdout.split() == [CHECKED, "True"]
    r = subprocess.run([sys.executable, "-m", "pytest", os.path.join(ROOT, "tests", "test_gpu_parity.py"), "-q",
                        "-m", "gpu", "-k", SELECTED, "-p", "no:cacheprovider"],
                       env=env, capture_output=True, text=True, timeout=1800, cwd=ROOT)
    assert r.returncode == 0, r.stdout[-4000:] + r.stderr[-2000:]
    assert " passed" in r.stdout and "failed" not in r.stdout
