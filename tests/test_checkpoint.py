"""Binary checkpoints (d3d_checkpoint_save / _load / _save_host), the
replacement for the reference's "%.7E" text dump (baseline.cc:62-70).

CPU: the host reader and writer of the format (benchmarks_b200
read_checkpoint / write_checkpoint) round-trip and reject a corrupted,
truncated or foreign file; d3d_checkpoint_save_host (no device work) writes
what the host reader reads.
GPU: device -> file -> host and host -> file -> device are bit-exact for 2D
and 3D, FP32 and FP64; the device rejects a wrong shape (D3D_E_INVALID), a
corrupted payload and a missing file (D3D_E_IO); a 512^3 field round-trips.
"""
import ctypes
import os

import numpy as np
import pytest

import benchmarks_b200 as B


@pytest.mark.parametrize("shape,dtype", [((5, 6, 7), np.float32),
                                         ((9, 130), np.float64),
                                         ((1, 1, 1), np.float32)])
def test_host_round_trip(tmp_path, shape, dtype):
    a = np.random.default_rng(1).random(shape).astype(dtype)
    p = str(tmp_path / "f.d3d")
    B.write_checkpoint(p, a, step=1234, diffusion_surface=len(shape) == 2)
    h, b = B.read_checkpoint(p)
    assert b.dtype == a.dtype and b.tobytes() == a.tobytes()
    assert h["step"] == 1234 and h["ndim"] == len(shape)
    assert h["flags"] == (1 if len(shape) == 2 else 0)
    assert os.path.getsize(p) == 64 + a.nbytes


def test_host_reader_rejects_damage(tmp_path):
    a = np.arange(1000, dtype=np.float32).reshape(10, 10, 10)
    p = str(tmp_path / "f.d3d")
    B.write_checkpoint(p, a)
    raw = bytearray(open(p, "rb").read())
    bad = bytearray(raw)
    bad[64 + 123] ^= 0x10
    open(p, "wb").write(bad)
    with pytest.raises(ValueError, match="checksum"):
        B.read_checkpoint(p)
    open(p, "wb").write(raw[:-4])
    with pytest.raises(ValueError, match="truncated"):
        B.read_checkpoint(p)
    open(p, "wb").write(b"NOTACKPT" + raw[8:])
    with pytest.raises(ValueError, match="not a d3d checkpoint"):
        B.read_checkpoint(p)


def test_save_host_through_the_c_abi(tmp_path):
    """d3d_checkpoint_save_host needs a plan only for its shape: a plan is
    created without touching a device when the arguments are rejected, so
    here the call is checked for its argument errors and, where a device
    exists, for the file it writes."""
    L = B.lib()
    assert L.d3d_checkpoint_save_host(None, None, 0, b"x") == B.D3D_E_INVALID
    assert L.d3d_checkpoint_save(None, None, 0, b"x", None) == B.D3D_E_INVALID
    assert L.d3d_checkpoint_load(None, b"x", None, None, None) \
        == B.D3D_E_INVALID


@pytest.mark.gpu
@pytest.mark.parametrize("dims,dtype", [((17, 23, 5), B.F32),
                                        ((40, 24, 12), B.F64),
                                        ((131, 37), B.F32),
                                        ((64, 64), B.F64)])
def test_device_round_trip(tmp_path, dims, dtype):
    import torch
    plan = (B.DiffusionPlan(dims, dtype) if len(dims) == 2
            else B.Plan(*dims, dtype))
    tdt = torch.float64 if dtype == B.F64 else torch.float32
    g = torch.Generator(device="cuda").manual_seed(3)
    f = torch.rand(plan.shape, device="cuda", dtype=tdt, generator=g)
    p = str(tmp_path / "f.d3d")
    plan.save_checkpoint(f, p, step=77)
    h, host = B.read_checkpoint(p)
    assert host.tobytes() == f.cpu().numpy().tobytes()
    assert h["step"] == 77 and (h["flags"] == 1) == (len(dims) == 2)
    back = plan.empty()
    assert plan.load_checkpoint(p, back) == 77
    assert torch.equal(back, f)
    # a host-written file goes to the device
    x = np.random.default_rng(5).random(plan.shape).astype(host.dtype)
    B.write_checkpoint(p, x, step=9, diffusion_surface=len(dims) == 2)
    assert plan.load_checkpoint(p, back) == 9
    assert back.cpu().numpy().tobytes() == x.tobytes()
    # the host form of the C ABI writes the same file as the device form
    q = str(tmp_path / "h.d3d")
    assert B.lib().d3d_checkpoint_save_host(
        plan.handle, x.ctypes.data_as(ctypes.c_void_p), 9,
        os.fsencode(q)) == 0
    plan.save_checkpoint(back, p, step=9)
    assert open(p, "rb").read() == open(q, "rb").read()
    plan.close()


@pytest.mark.gpu
def test_device_load_rejects_wrong_shape_and_damage(tmp_path):
    plan = B.Plan(16, 16, 8)
    p = str(tmp_path / "f.d3d")
    B.write_checkpoint(p, np.zeros((8, 16, 17), np.float32))
    buf = plan.empty()
    with pytest.raises(B.D3DError) as ei:
        plan.load_checkpoint(p, buf)
    assert ei.value.code == B.D3D_E_INVALID
    a = np.random.default_rng(2).random((8, 16, 16)).astype(np.float32)
    B.write_checkpoint(p, a)
    raw = bytearray(open(p, "rb").read())
    raw[64 + 4 * 1000 + 2] ^= 0x01
    open(p, "wb").write(raw)
    with pytest.raises(B.D3DError) as ei:
        plan.load_checkpoint(p, buf)
    assert ei.value.code == B.D3D_E_IO
    with pytest.raises(B.D3DError) as ei:
        plan.load_checkpoint(str(tmp_path / "missing.d3d"), buf)
    assert ei.value.code == B.D3D_E_IO
    # Same shape, saved from the diffusion::Diffusion surface (y order
    # flipped): refused before the field is touched.
    B.write_checkpoint(p, a, diffusion_surface=True)
    buf.fill_(7.0)
    with pytest.raises(B.D3DError) as ei:
        plan.load_checkpoint(p, buf)
    assert ei.value.code == B.D3D_E_INVALID
    assert "diffusion::Diffusion" in str(ei.value)
    assert bool((buf == 7.0).all())
    assert B.check_device_errors() == 0
    plan.close()


@pytest.mark.gpu
def test_full_size_round_trip(tmp_path):
    """A 512^3 FP32 field (512 MiB, 8 staging chunks) out and back."""
    import torch
    plan = B.Plan(512, 512, 512)
    g = torch.Generator(device="cuda").manual_seed(4)
    f = torch.rand(plan.shape, device="cuda", generator=g)
    p = str(tmp_path / "big.d3d")
    plan.save_checkpoint(f, p, step=200)
    assert os.path.getsize(p) == 64 + 512 ** 3 * 4
    back = plan.empty()
    assert plan.load_checkpoint(p, back) == 200
    assert torch.equal(back, f)
    os.remove(p)
    plan.close()
