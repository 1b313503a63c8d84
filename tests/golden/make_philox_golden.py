"""Generates tests/golden/philox_curand.json: device cuRAND Philox4_32_10 output (seed 1234) for a
set of subsequences, captured on a B200 through tests/kat/libphilox_kat.so. The CPU test suite
checks the oracle's Philox stream against these vectors without a GPU.

Usage (on a machine with a CUDA device): python tests/golden/make_philox_golden.py [output.json]
"""
import ctypes
import json
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
KAT = os.path.join(os.path.dirname(HERE), "kat")
SUBSEQUENCES = [0, 1, 2, 3, 7, 1000, 65535, 123456789, 2**32 + 5, 2**40 + 77, 132710399]


def main(out_path):
    import torch
    lib_path = os.path.join(KAT, "libphilox_kat.so")
    if not os.path.exists(lib_path):
        subprocess.run(["make", "-s", "-C", KAT], check=True)
    L = ctypes.CDLL(lib_path)
    L.philox_kat.restype = ctypes.c_int
    L.philox_kat.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                             ctypes.c_void_p]
    n = len(SUBSEQUENCES)
    s = torch.tensor(np.asarray(SUBSEQUENCES, dtype=np.uint64).view(np.int64), device="cuda")
    o = torch.zeros(1, dtype=torch.int32, device="cuda")
    sched = torch.zeros((n, 14), dtype=torch.float32, device="cuda")
    reinit = torch.zeros((n, 1, 4), dtype=torch.float32, device="cuda")
    words = torch.zeros((n, 8), dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    assert L.philox_kat(s.data_ptr(), n, o.data_ptr(), 1, sched.data_ptr(), reinit.data_ptr(), words.data_ptr()) == 0
    sched_np = sched.cpu().numpy()
    words_np = words.cpu().numpy().view(np.uint32)
    records = [{"subsequence": int(sub), "words": [int(w) for w in words_np[i]],
                "schedule": [float(v) for v in sched_np[i]]} for i, sub in enumerate(SUBSEQUENCES)]
    doc = {"generator": "curand_init(1234, subsequence, 0); curand4 x2 (words); uniform4, uniform4, uniform, uniform4, "
                        "uniform (schedule)", "device": torch.cuda.get_device_name(0), "records": records}
    with open(out_path, "w") as f:
        json.dump(doc, f, indent=1)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(HERE, "philox_curand.json"))
