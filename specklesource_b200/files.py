"""Reference file formats used by the drop-in tools (strack/strackw/cullst).

SLC images are raw row-major complex samples (big-endian float32 by default,
or complex int16) described by a GDAL VRT sidecar; parameter files are RDF
"key = value" lines (Strack/parseTrack.c); offsets grids are raw float32
files (.dr .da .cc .azd), uint8 match types (.mt) and a one-line .dat header
(writeDatFile, Strack/speckleTrack.c:1453-1469).
"""
import os

import numpy as np

# the keys parseTrack reads, in its order
TRACK_KEYS = ("image1", "image2", "outputfile", "initialoffsetfile", "initShift", "intfile", "intgeodat", "baseparams",
              "offsetmaskfile", "offsetmaskdat", "rstart", "astart", "deltar", "deltaa", "nR", "nA", "wr", "wa",
              "wra", "waa", "edgepad", "scalefactor", "navgR", "navgA")


def write_slc(path, img, byte_order="MSB"):
    """Writes a complex image as raw samples plus <path>.vrt (CFloat32 or CInt16)."""
    if np.iscomplexobj(img):
        data = np.ascontiguousarray(img, dtype=">c8" if byte_order == "MSB" else "<c8")
        dtype = "CFloat32"
        pix = 8
    else:  # int16 (na, nr, 2)
        data = np.ascontiguousarray(img, dtype=">i2" if byte_order == "MSB" else "<i2")
        dtype = "CInt16"
        pix = 4
    na, nr = data.shape[:2]
    data.tofile(path)
    with open(path + ".vrt", "w") as f:
        f.write(f'<VRTDataset rasterXSize="{nr}" rasterYSize="{na}">\n'
                f'  <VRTRasterBand dataType="{dtype}" band="1" subClass="VRTRawRasterBand">\n'
                f'    <SourceFilename relativeToVRT="1">{os.path.basename(path)}</SourceFilename>\n'
                f'    <ImageOffset>0</ImageOffset>\n    <PixelOffset>{pix}</PixelOffset>\n'
                f'    <LineOffset>{nr * pix}</LineOffset>\n    <ByteOrder>{byte_order}</ByteOrder>\n'
                f'  </VRTRasterBand>\n</VRTDataset>\n')


def write_interferogram(path, data, nrl, nal, lines=None):
    """Complex int16 interferogram (na, nr, 2) as the strack tool reads it:
    raw samples (byte order of the array) plus <path>.vrt giving the size, the
    byte order and the looks (metadata nRangeLooks / nAzimuthLooks).  lines:
    write only the first `lines` rows (a short file)."""
    data = np.ascontiguousarray(data)
    na, nr = data.shape[:2]
    order = "MSB" if data.dtype.byteorder == ">" else "LSB"
    (data if lines is None else data[:lines]).tofile(path)
    with open(path + ".vrt", "w") as f:
        f.write(f'<VRTDataset rasterXSize="{nr}" rasterYSize="{na}">\n'
                f'  <Metadata>\n    <MDI key="nRangeLooks">{nrl}</MDI>\n'
                f'    <MDI key="nAzimuthLooks">{nal}</MDI>\n  </Metadata>\n'
                f'  <VRTRasterBand dataType="CInt16" band="1" subClass="VRTRawRasterBand">\n'
                f'    <SourceFilename relativeToVRT="1">{os.path.basename(path)}</SourceFilename>\n'
                f'    <ImageOffset>0</ImageOffset>\n    <PixelOffset>4</PixelOffset>\n'
                f'    <LineOffset>{nr * 4}</LineOffset>\n    <ByteOrder>{order}</ByteOrder>\n'
                f'  </VRTRasterBand>\n</VRTDataset>\n')


def write_poly(path, r=(0.0, 0.0, 0.0), a=(0.0, 0.0, 0.0)):
    """Initial-offset polynomial file (parseInitialOffsets.c:40-57)."""
    with open(path, "w") as f:
        f.write(f"range_offset_polynomial: {r[0]} {r[1]} {r[2]}\n")
        f.write(f"azimuth_offset_polynomial: {a[0]} {a[1]} {a[2]}\n")


def write_parfile(path, **kv):
    """RDF parameter file with units and comments, as GrIMP writes them."""
    with open(path, "w") as f:
        f.write("; speckle tracking parameters\n")
        for k, v in kv.items():
            unit = " (pixels)" if k in ("rstart", "astart", "deltar", "deltaa", "wr", "wa", "wra", "waa") else ""
            f.write(f"{k}{unit} = {v}   ! {k}\n")


def read_grid(path, nr, na, dtype=np.float32, byte_order="MSB"):
    dt = np.dtype(dtype).newbyteorder(">" if byte_order == "MSB" and np.dtype(dtype).itemsize > 1 else "=")
    return np.fromfile(path, dtype=dt, count=nr * na).reshape(na, nr).astype(dtype)


def read_track_outputs(base, nr, na, byte_order="MSB", azd=True):
    out = {k: read_grid(f"{base}.{k}", nr, na, np.float32, byte_order) for k in ("dr", "da", "cc")}
    if azd:
        out["azd"] = read_grid(f"{base}.azd", nr, na, np.float32, byte_order)
    out["mt"] = read_grid(f"{base}.mt", nr, na, np.uint8)
    return out


def write_offsets(base, offR, offA, corr, mt, r0, a0, deltaR, deltaA):
    """cullst input: <base>.{dr,da,cc,mt} (MSB) and <base>.dat."""
    na, nr = offR.shape
    np.ascontiguousarray(offR, ">f4").tofile(base + ".dr")
    np.ascontiguousarray(offA, ">f4").tofile(base + ".da")
    np.ascontiguousarray(corr, ">f4").tofile(base + ".cc")
    np.ascontiguousarray(mt, np.uint8).tofile(base + ".mt")
    with open(base + ".dat", "w") as f:
        f.write(f"{r0} {a0} {nr} {na} {deltaR} {deltaA}\n")
