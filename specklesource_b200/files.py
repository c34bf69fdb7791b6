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


def write_ls_culled(match_file, res, params, meta):
    """writeLSCulledOffsets (Cullls/cullls.c:61-161): <match_file>.cull.dx,
    .cull.dy, .cull.sx, .cull.sy (big-endian float32), .cull.mtype (uint8) and
    the .cull.dat summary.  res: a cullls result (XS, YS, sigmaX, sigmaY,
    type, nMatch, nAttempt); params: its CullLSParams (noDataLimit); meta: the
    matchResult/lsFit fields the summary prints (fileEarly, fileLate, x0, y0,
    dx, dy, stepX, stepY, slowFlag, proj, jdEarly, jdLate).  Returns the
    summary's (nGoodPts, sigmaXAvg, sigmaYAvg)."""
    XS, YS = res["XS"], res["YS"]
    ny, nx = XS.shape
    good = (XS.astype(np.float64) > params.noDataLimit) & (YS.astype(np.float64) > params.noDataLimit)
    n_good = int(good.sum())
    # float products summed in double in raster order, as the reference's loop
    sx = res["sigmaX"][good].astype(np.float32)
    sy = res["sigmaY"][good].astype(np.float32)
    acc_x = float(np.cumsum((sx * sx).astype(np.float64))[-1]) if n_good else 0.0
    acc_y = float(np.cumsum((sy * sy).astype(np.float64))[-1]) if n_good else 0.0
    sig_x = float(np.sqrt(acc_x / max(n_good, 1)))
    sig_y = float(np.sqrt(acc_y / max(n_good, 1)))
    for ext, arr in ((".cull.dx", XS), (".cull.dy", YS), (".cull.sx", res["sigmaX"]), (".cull.sy", res["sigmaY"])):
        np.ascontiguousarray(arr, ">f4").tofile(match_file + ext)
    np.ascontiguousarray(res["type"], np.uint8).tofile(match_file + ".cull.mtype")
    att = max(int(res["nAttempt"]), 1)
    success = float(np.float32(res["nMatch"]) / np.float32(att)) * 100.0
    culled = float(np.float32(n_good) / np.float32(att)) * 100.0
    m = meta
    lines = [
        f"fileEarly = {m['fileEarly']}",
        f"fileLate = {m['fileLate']}",
        f"x0 = {m['x0']:11.2f}",
        f"y0 = {m['y0']:11.2f}",
        f"dx = {m['dx']:10.5f}",
        f"dy = {m['dy']:10.5f}",
        f"stepY = {int(m['stepX'])}",  # the reference prints stepX under "stepY" and vice versa
        f"stepX = {int(m['stepY'])}",
        f"nx = {nx:9d}",
        f"ny = {ny:9d}",
        f"slowFlag = {int(m['slowFlag']):9d}",
        f"EPSG = {int(m['proj']):9d}",
        f"earlyImageJD = {m['jdEarly']:10f}",
        f"lateImageJD = {m['jdLate']:10f}",
        f"IntervalBetweenImages = {int(m['jdLate'] - m['jdEarly']):5d}",
        f"Success_rate_for_attempted_matches(%) =  {success:7.2f} ",
        f"Culled_rate_for_attempted_matches(%) =  {culled:7.2f} ",
        f"Mean_sigmaX = {sig_x:11.3f}",
        f"Mean_sigmaY = {sig_y:11.3f}",
        "& ",
    ]
    with open(match_file + ".cull.dat", "w") as f:
        f.write("\n".join(lines) + "\n")
    return n_good, sig_x, sig_y
