"""bench.py's reference arm (the CPU restatement timed on the host cores) prints one JSON line
with the keys the benchmark contract asks for (CPU; a tiny sample)."""
import json
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def test_reference_arm_json_line():
    out = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--nmol", "16", "--steps", "1",
                          "--warmup", "1"], capture_output=True, text=True, timeout=300,
                         check=True).stdout.strip().splitlines()
    assert len(out) == 1
    d = json.loads(out[0])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "higher_is_better", "scaling", "dtype",
                "data", "config", "cpu_baseline", "e2e", "impl"):
        assert key in d, key
    assert d["impl"] == "reference" and d["unit"] == "mol/s" and d["value"] > 0
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    assert d["config"]["sample_per_step"] == 16  # the whole (tiny) batch each step


def test_cpu_samples_keep_both_kinds_of_molecule():
    """The mixed batch alternates water clusters and alkanes; every CPU sample (each step's
    offset) holds both kinds in equal numbers and the batch's size distribution."""
    sys.path.insert(0, str(ROOT))
    import numpy as np

    import bench
    from axtb_b200 import structures
    from axtb_b200.calculator import basis_size

    mols = structures.mixed_batch(1024, seed=0)
    n2 = np.mean([float(basis_size(z)[1]) ** 2 for z, _ in mols])
    for offset in range(4):
        sample = bench.interleaved(mols, 64, offset)
        waters = sum(1 for z, _ in sample if 6 not in z)
        assert len(sample) == 64 and waters == 32
        s2 = np.mean([float(basis_size(z)[1]) ** 2 for z, _ in sample])
        assert 0.6 < s2 / n2 < 1.4
