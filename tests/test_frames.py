"""Frame output (fmm_frames_*), the counterpart of the reference's
HDF5Exporter (io/hdf5_exporter.cpp): the datasets of write_frame and the
XDMF temporal index of write_xdmf_metadata, here with the datasets as raw
little-endian FP64 in one .bin per frame.  CPU tests write from host
arrays; the GPU tests write from device arrays through the asynchronous
path and expect the same bytes, and check the integrator loop's frames
against the states of plain integrator runs."""
import os
import subprocess

import numpy as np
import pytest
from conftest import ROOT

import fmmgpu


def expected_index(frames):
    """The reference's index text (hdf5_exporter.cpp:88-127) for frames
    [(time, file, n)], with each data item pointing into the frame's .bin
    (Format="Binary", Seek = byte offset of the dataset)."""
    out = ['<?xml version="1.0" ?>\n', '<!DOCTYPE Xdmf SYSTEM "Xdmf.dtd" []>\n', '<Xdmf Version="2.0">\n',
           ' <Domain>\n', '  <Grid Name="TimeSeries" GridType="Collection" CollectionType="Temporal">\n']

    def item(dims, seek, f):
        return [f'       <DataItem Dimensions="{dims}" NumberType="Float" Precision="8" Format="Binary" '
                f'Endian="Little" Seek="{seek}">\n', f'         {f}\n', '       </DataItem>\n']

    for t, (time, f, n) in enumerate(frames):
        out += [f'   <Grid Name="Step_{t}" GridType="Uniform">\n', f'     <Time Value="{time:g}"/>\n',
                f'     <Topology TopologyType="Polyvertex" NumberOfElements="{n}"/>\n',
                '     <Geometry GeometryType="XYZ">\n', *item(f"{n} 3", 0, f), '     </Geometry>\n',
                '     <Attribute Name="Velocity" AttributeType="Vector" Center="Node">\n', *item(f"{n} 3", 24 * n, f),
                '     </Attribute>\n',
                '     <Attribute Name="Acceleration" AttributeType="Vector" Center="Node">\n',
                *item(f"{n} 3", 48 * n, f), '     </Attribute>\n',
                '     <Attribute Name="Weight" AttributeType="Scalar" Center="Node">\n', *item(f"{n}", 72 * n, f),
                '     </Attribute>\n', '   </Grid>\n']
    out += ['  </Grid>\n', ' </Domain>\n', '</Xdmf>\n']
    return "".join(out)


def read_frame(path, n):
    a = np.fromfile(path, dtype="<f8")
    assert a.size == 10 * n
    return a[:3 * n].reshape(n, 3), a[3 * n:6 * n].reshape(n, 3), a[6 * n:9 * n].reshape(n, 3), a[9 * n:]


def pad3(x):
    return np.hstack([x, np.zeros((len(x), 3 - x.shape[1]))]) if x.shape[1] < 3 else x


def system(n, dim, seed):
    rng = np.random.default_rng(seed)
    return rng.normal(size=(n, dim)), rng.normal(size=(n, dim)), rng.normal(size=(n, dim)), rng.uniform(1, 2, n)


@pytest.mark.parametrize("dim", [3, 2])
def test_frames_hold_the_reference_datasets_and_index(tmp_path, dim):
    d = tmp_path / "out"
    frames, want = [], []
    with fmmgpu.Frames(str(d), "particles", dim=dim) as fr:
        for step, (n, time) in enumerate([(1000, 0.0), (1000, 0.001), (0, 0.002), (700, 1e-05)]):
            pos, vel, acc, m = system(n, dim, step)
            fr.write(pos, vel, m, step, time, acc=None if step == 1 else acc)
            if n == 0:  # an empty frame is skipped (hdf5_exporter.cpp:22)
                assert not (d / f"particles_{step:05d}.bin").exists()
                continue
            name = f"particles_{step:05d}.bin"
            frames.append((time, name, n))
            want.append((name, n, pad3(pos), pad3(vel), np.zeros((n, 3)) if step == 1 else pad3(acc), m))
            # the index is rewritten after every frame
            assert (d / "particles.xmf").read_text() == expected_index(frames)
    for name, n, pos, vel, acc, m in want:
        p, v, a, w = read_frame(d / name, n)
        np.testing.assert_array_equal(p, pos)
        np.testing.assert_array_equal(v, vel)
        np.testing.assert_array_equal(a, acc)
        np.testing.assert_array_equal(w, m)


def test_frames_errors(tmp_path):
    with pytest.raises(fmmgpu.FmmError) as e:
        fmmgpu.Frames(str(tmp_path), dim=4)
    assert e.value.code == fmmgpu.FMM_ERR_INVALID_ARGUMENT
    blocker = tmp_path / "file"
    blocker.write_text("x")
    with pytest.raises(fmmgpu.FmmError) as e:
        fmmgpu.Frames(str(blocker / "sub"))
    assert e.value.code == fmmgpu.FMM_ERR_IO


def test_exporter_drop_in_for_the_reference_driver(tmp_path):
    """GpuFrameExporter (nbody-fmm_b200/cpp/gpu_fmm.hpp), HDF5Exporter's
    interface, compiled against the reference's Particle: three frames of
    the reference's own particles, datasets checked by the program itself
    (oracle/adapter_check.cpp), the index here."""
    exe = os.path.join(ROOT, "oracle", "_ref", "adapter_check")
    if not os.path.exists(exe):
        pytest.skip("the reference is not built here (oracle/_ref)")
    r = subprocess.run([exe, "frames", str(tmp_path)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr[-2000:]
    want = [(0.5 * k, f"particles_{k:05d}.bin", 50) for k in range(3)]
    assert (tmp_path / "particles.xmf").read_text() == expected_index(want)


@pytest.mark.gpu
def test_device_frames_match_host_frames(tmp_path):
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda", 0)
    n, dim = 5000, 3
    systems = [system(n, dim, s) for s in range(4)]
    with fmmgpu.Frames(str(tmp_path / "host"), dim=dim) as fh:
        for step, (pos, vel, acc, m) in enumerate(systems):
            fh.write(pos, vel, m, step, 0.5 * step, acc=acc)
    st = torch.cuda.Stream(dev)
    with fmmgpu.Frames(str(tmp_path / "dev"), dim=dim) as fd:
        keep = []
        for step, (pos, vel, acc, m) in enumerate(systems):
            t = [torch.from_numpy(x).to(dev) for x in (pos, vel, acc, m)]
            torch.cuda.synchronize()
            keep.append(t)  # device arrays stay alive until their copy has run
            fd.write_device(n, t[0].data_ptr(), t[1].data_ptr(), t[3].data_ptr(), step, 0.5 * step,
                            acc_ptr=t[2].data_ptr(), stream=st.cuda_stream)
        fd.flush()
    for step in range(4):
        name = f"particles_{step:05d}.bin"
        assert (tmp_path / "dev" / name).read_bytes() == (tmp_path / "host" / name).read_bytes()
    assert (tmp_path / "dev" / "particles.xmf").read_text() == (tmp_path / "host" / "particles.xmf").read_text()


@pytest.mark.gpu
def test_integrate_frames_writes_the_state_before_each_step(tmp_path):
    """The reference's loop (main.cpp:85-91): frame k is the state after k
    steps, with the acceleration of the last force evaluation (zeros before
    the first step); checked against plain fmm_integrate runs of k steps."""
    from fmmgpu import workloads

    n, dt, steps = 2000, 1e-3, 3
    pos0, m = workloads.plummer(n, seed=8)
    vel0 = np.zeros_like(pos0)
    with fmmgpu.Context(dim=3, p=8, leaf_cap=64, G=1.0) as c:
        with fmmgpu.Frames(str(tmp_path), dim=3) as fr:
            c.integrate(fmmgpu.FMM_INT_SYMPLECTIC_EULER, dt, steps, pos0, vel0, m, frames=fr, every=1, step0=10,
                        t0=0.5)
        want = [(pos0, vel0, np.zeros_like(pos0))]
        for k in range(1, steps):
            want.append(c.integrate(fmmgpu.FMM_INT_SYMPLECTIC_EULER, dt, k, pos0, vel0, m))
    for k, (wp, wv, wa) in enumerate(want):
        p, v, a, w = read_frame(tmp_path / f"particles_{10 + k:05d}.bin", n)
        np.testing.assert_allclose(p, wp, rtol=1e-6, atol=1e-12)
        np.testing.assert_allclose(v, wv, rtol=1e-6, atol=1e-9)
        np.testing.assert_allclose(a, wa, rtol=1e-6, atol=1e-6 * np.abs(wa).max() + 1e-300)
        np.testing.assert_array_equal(w, m)
    idx = (tmp_path / "particles.xmf").read_text()
    assert idx == expected_index([(0.5 + k * dt, f"particles_{10 + k:05d}.bin", n) for k in range(steps)])
