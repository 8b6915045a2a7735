"""The device closure (cenote_b200/csrc/openpbr.cuh) compiled for the host
through tests/host/cuda_host_shim.h, in FP32, against the FP64 oracle — the
same budgets as the GPU test, checked without a GPU."""
import pathlib
import subprocess

import numpy as np
import pytest

import oracle
from test_gpu_parity import directions, materials, rel_err
from test_traversal_host import CSRC, HOST, cuda_include


@pytest.fixture(scope="module")
def bsdf_host(tmp_path_factory):
    d = tmp_path_factory.mktemp("bsdf")
    exe = d / "bsdf_host"
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", f"-I{HOST}", f"-I{CSRC}", f"-I{cuda_include()}",
                    "-include", str(HOST / "cuda_host_shim.h"), str(HOST / "bsdf_host.cpp"), "-o", str(exe)],
                   check=True)
    oracle.bsdf_tables().tofile(d / "tables.bin")

    def run(mat, wo, wi, exiting):
        np.asarray(mat).tofile(d / "m.bin")
        np.concatenate([wo, wi], 1).astype(np.float32).tofile(d / "dirs.bin")
        subprocess.run([str(exe), str(d / "tables.bin"), str(d / "m.bin"), str(d / "dirs.bin"), "1" if exiting else "0",
                        str(d / "out.bin")], check=True)
        o = np.fromfile(d / "out.bin", np.float32).reshape(-1, 4)
        return o[:, :3], o[:, 3]

    return run


@pytest.mark.parametrize("name", list(materials()))
@pytest.mark.parametrize("exiting", [False, True])
def test_device_closure_on_host_vs_fp64(bsdf_host, name, exiting):
    mat = materials()[name]
    wo, wi = directions(20000, seed=sum(map(ord, name)))
    f, pdf = bsdf_host(mat, wo, wi, exiting)
    rf, rpdf = oracle.bsdf_eval(mat, wo, wi, exiting)
    e = np.maximum(rel_err(f.astype(np.float64), rf, 1e-2).max(axis=1), rel_err(pdf.astype(np.float64), rpdf, 1e-2))
    frac_budget, worst = (1e-2, 2e-3) if exiting else (1e-3, 1e-4)
    assert (e > 1e-5).mean() <= frac_budget and e.max() <= worst, (name, exiting, np.sort(e)[-3:])
