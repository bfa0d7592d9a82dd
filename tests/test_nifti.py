"""NIfTI-1 input / output (claire_b200_read_nifti / _write_nifti), host only.

Files are produced and parsed here by an independent writer / reader of the
published NIfTI-1 single-file layout (348-byte header, 4-byte extension flag,
voxels at vox_offset, x fastest), so the library is checked against the
format, not against itself.  The grid mapping follows ReadWriteReg::ReadNII
(src/ReadWriteReg.cpp:813-815): CLAIRE's nx = (nz, ny, nx) of the file.
"""
import gzip
import os
import struct

import numpy as np
import pytest

# directory of the reference's example images (doc/data/brain0{1,2}.nii.gz);
# the test that reads them is skipped when it is not set or not present
REF_DATA = os.environ.get("CLAIRE_EXAMPLE_DATA", "")

DTYPES = {2: np.uint8, 256: np.int8, 4: np.int16, 512: np.uint16, 8: np.int32, 768: np.uint32, 16: np.float32,
          64: np.float64}


def make_nifti(vol_xyz_order, code, big_endian=False, vox_offset=352, extra_dims=()):
    """Bytes of a single-file NIfTI-1 image; vol is indexed [z][y][x] (x fastest)."""
    bo = ">" if big_endian else "<"
    nz, ny, nx = vol_xyz_order.shape
    dims = [3 + len(extra_dims), nx, ny, nz] + list(extra_dims)
    dims += [1] * (8 - len(dims))
    h = bytearray(348)
    struct.pack_into(bo + "i", h, 0, 348)
    struct.pack_into(bo + "8h", h, 40, *dims)
    dt = np.dtype(DTYPES[code]).newbyteorder(bo)
    struct.pack_into(bo + "h", h, 70, code)
    struct.pack_into(bo + "h", h, 72, dt.itemsize * 8)
    struct.pack_into(bo + "8f", h, 76, 1, 1, 1, 1, 1, 1, 1, 1)
    struct.pack_into(bo + "f", h, 108, float(vox_offset))
    struct.pack_into(bo + "f", h, 112, 2.0)  # scl_slope: not applied (ReadNII casts raw values)
    h[344:348] = b"n+1\0"
    pad = bytes(vox_offset - 348)
    count = int(np.prod(extra_dims)) if extra_dims else 1
    data = np.concatenate([vol_xyz_order.ravel()] * count).astype(dt).tobytes()
    return bytes(h) + pad + data


def parse_nifti(raw):
    h = raw[:348]
    assert struct.unpack_from("<i", h, 0)[0] == 348
    dims = struct.unpack_from("<8h", h, 40)
    code = struct.unpack_from("<h", h, 70)[0]
    pixdim = struct.unpack_from("<8f", h, 76)
    off = int(struct.unpack_from("<f", h, 108)[0])
    assert h[344:348] == b"n+1\0"
    n = dims[1] * dims[2] * dims[3]
    data = np.frombuffer(raw, dtype=np.dtype(DTYPES[code]).newbyteorder("<"), count=n, offset=off)
    return dims, code, pixdim, data.reshape(dims[3], dims[2], dims[1])


@pytest.fixture(scope="module")
def cb():
    import claire_b200
    return claire_b200


@pytest.mark.parametrize("code", sorted(DTYPES))
@pytest.mark.parametrize("gz", [False, True])
def test_read_every_type_and_both_compressions(cb, tmp_path, code, gz):
    rng = np.random.default_rng(code)
    vol = (rng.uniform(0, 100, size=(5, 6, 7))).astype(DTYPES[code])  # (nz, ny, nx)
    raw = make_nifti(vol, code)
    p = tmp_path / ("v.nii.gz" if gz else "v.nii")
    p.write_bytes(gzip.compress(raw) if gz else raw)
    out = cb.read_nifti(str(p))
    assert out.shape == (5, 6, 7) and out.dtype == np.float32
    assert np.array_equal(out, vol.astype(np.float32))


def test_big_endian_and_offset(cb, tmp_path):
    vol = np.arange(4 * 3 * 2, dtype=np.int16).reshape(4, 3, 2) - 7
    p = tmp_path / "be.nii"
    p.write_bytes(make_nifti(vol, 4, big_endian=True, vox_offset=400))
    assert np.array_equal(cb.read_nifti(str(p)), vol.astype(np.float32))


def test_write_then_read_and_parse(cb, tmp_path):
    rng = np.random.default_rng(1)
    vol = rng.standard_normal((8, 9, 10)).astype(np.float32)
    for name in ("w.nii", "w.nii.gz"):
        p = str(tmp_path / name)
        cb.write_nifti(p, vol)
        raw = open(p, "rb").read()
        if name.endswith(".gz"):
            assert raw[:2] == b"\x1f\x8b"
            raw = gzip.decompress(raw)
        dims, code, pixdim, data = parse_nifti(raw)
        # AllocateImage: 5 dims, (nx, ny, nz) = (nx[2], nx[1], nx[0]), float32
        assert dims[:6] == (5, 10, 9, 8, 1, 1) and code == 16
        assert abs(pixdim[1] - 2 * np.pi / 8) < 1e-6
        assert np.array_equal(data, vol)
        assert np.array_equal(cb.read_nifti(p), vol)


def test_unsupported_and_missing(cb, tmp_path):
    vol = np.zeros((2, 2, 2), np.float32)
    p = tmp_path / "t.nii"
    p.write_bytes(make_nifti(vol, 16, extra_dims=(2,)))  # two time points
    with pytest.raises(cb.ClaireError):
        cb.read_nifti(str(p))
    with pytest.raises(cb.ClaireError):
        cb.read_nifti(str(tmp_path / "missing.nii"))


@pytest.mark.skipif(not REF_DATA or not os.path.isdir(REF_DATA),
                    reason="CLAIRE_EXAMPLE_DATA does not name the reference's example images")
@pytest.mark.parametrize("name", ["brain01.nii.gz", "brain02.nii.gz"])
def test_reference_example_brains(cb, name):
    path = os.path.join(REF_DATA, name)
    raw = gzip.decompress(open(path, "rb").read())
    h = raw[:348]
    bo = "<" if struct.unpack_from("<i", h, 0)[0] == 348 else ">"
    dims = struct.unpack_from(bo + "8h", h, 40)
    code = struct.unpack_from(bo + "h", h, 70)[0]
    off = int(struct.unpack_from(bo + "f", h, 108)[0])
    n = dims[1] * dims[2] * dims[3]
    ref = np.frombuffer(raw, dtype=np.dtype(DTYPES[code]).newbyteorder(bo), count=n, offset=off)
    out = cb.read_nifti(path)
    assert out.shape == (dims[3], dims[2], dims[1])
    assert np.array_equal(out.ravel(), ref.astype(np.float32))


def test_two_file_pair_read_and_write(cb, tmp_path):
    # NIfTI-1 pair (NIFTI_FTYPE_NIFTI1_2, src/ReadWriteReg.cpp:1305-1306):
    # header with magic "ni1" in .hdr, voxels at vox_offset (0) of .img
    rng = np.random.default_rng(7)
    vol = rng.uniform(-5, 5, size=(4, 5, 6)).astype(np.float32)  # (nz, ny, nx)
    single = make_nifti(vol, 16)
    h = bytearray(single[:348])
    h[344:348] = b"ni1\0"
    struct.pack_into("<f", h, 108, 0.0)
    for gz in (False, True):
        suf = ".gz" if gz else ""
        hdr, img = tmp_path / f"p.hdr{suf}", tmp_path / f"p.img{suf}"
        data = vol.tobytes()
        hdr.write_bytes(gzip.compress(bytes(h)) if gz else bytes(h))
        img.write_bytes(gzip.compress(data) if gz else data)
        for name in (hdr, img):
            assert np.array_equal(cb.read_nifti(str(name)), vol)
    # writing a pair: .hdr with "ni1" and vox_offset 0, .img with the voxels
    cb.write_nifti(str(tmp_path / "w.hdr"), vol)
    raw_h = (tmp_path / "w.hdr").read_bytes()
    assert raw_h[344:348] == b"ni1\0" and struct.unpack_from("<f", raw_h, 108)[0] == 0.0
    assert struct.unpack_from("<8h", raw_h, 40)[:4] == (5, 6, 5, 4)
    assert np.array_equal(np.frombuffer((tmp_path / "w.img").read_bytes(), dtype="<f4").reshape(vol.shape), vol)
    assert np.array_equal(cb.read_nifti(str(tmp_path / "w.img")), vol)
    # a pair header without its .img name is refused
    (tmp_path / "lone.nii").write_bytes(bytes(h))
    with pytest.raises(cb.ClaireError):
        cb.read_nifti(str(tmp_path / "lone.nii"))


def test_petsc_binary_vectors(cb, tmp_path):
    # ReadBIN / WriteBIN (src/ReadWriteReg.cpp:1476-1535): VecView / VecLoad
    # layout, big-endian class id 1211214, length, values
    rng = np.random.default_rng(8)
    vol = rng.standard_normal((3, 4, 5)).astype(np.float32)
    p = tmp_path / "v.bin"
    cb.write_image(str(p), vol)
    raw = p.read_bytes()
    cid, n = struct.unpack_from(">ii", raw, 0)
    assert cid == 1211214 and n == vol.size and len(raw) == 8 + 8 * n
    assert np.array_equal(np.frombuffer(raw, dtype=">f8", offset=8).astype(np.float32).reshape(vol.shape), vol)
    assert np.array_equal(cb.read_image(str(p), vol.shape), vol)
    # a single-precision build's file: 4-byte values
    q = tmp_path / "s.bin"
    q.write_bytes(struct.pack(">ii", 1211214, vol.size) + vol.astype(">f4").tobytes())
    assert np.array_equal(cb.read_bin(str(q), vol.shape), vol)
    # the length must match the grid; the class id must be a vector's
    with pytest.raises(cb.ClaireError):
        cb.read_bin(str(q), (3, 4, 6))
    bad = tmp_path / "bad.bin"
    bad.write_bytes(struct.pack(">ii", 1211215, vol.size) + vol.astype(">f4").tobytes())
    with pytest.raises(cb.ClaireError):
        cb.read_bin(str(bad), vol.shape)
    with pytest.raises(ValueError):
        cb.read_image(str(p))
