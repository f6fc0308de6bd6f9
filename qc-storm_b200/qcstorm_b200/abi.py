"""ctypes mirror of the qcstorm_b200 C ABI (include/qcstorm_b200.h).

`LocPara` has the field names, types and order of the reference's
LocalizationPara (bfgs_base.h:26-99) and of `qcs_loc_para`.
"""
import ctypes as C
import os

_FIELDS = [
    ("Offset", C.c_float), ("KAdc", C.c_float), ("QE", C.c_float), ("ReadNoise_e", C.c_float),
    ("ROISize", C.c_int), ("LocType", C.c_int), ("MultiEmitterFitEn", C.c_int), ("WLEEn", C.c_int),
    ("ConsecFit_DistanceTh_nm", C.c_float), ("ConsecFitEn", C.c_int),
    ("PixelSize", C.c_float), ("PixelZoom", C.c_float), ("SNR_th", C.c_float), ("ColorMode_3D", C.c_int),
    ("ImageWidth", C.c_int), ("ImageHigh", C.c_int), ("TotalFrameNum", C.c_int),
    ("SRImageWidth", C.c_int), ("SRImageHigh", C.c_int),
    ("MinZDepth", C.c_float), ("MaxZDepth", C.c_float), ("ZDepthCorrFactor", C.c_float),
    ("p4_XGY", C.c_float), ("p3_XGY", C.c_float), ("p2_XGY", C.c_float), ("p1_XGY", C.c_float), ("p0_XGY", C.c_float),
    ("p4_XLY", C.c_float), ("p3_XLY", C.c_float), ("p2_XLY", C.c_float), ("p1_XLY", C.c_float), ("p0_XLY", C.c_float),
    ("DH_RotateType", C.c_int), ("DH_MeanDistance", C.c_float), ("DH_DistanceTh", C.c_float),
    ("ImagesPerGroup", C.c_int), ("IsHollowTube", C.c_int), ("StrucuteSize_2D", C.c_float),
    ("SpatialResolutionCalcEn", C.c_int),
]


class LocPara(C.Structure):
    _fields_ = _FIELDS

    def copy(self, **changes):
        out = LocPara()
        C.pointer(out)[0] = self
        for k, v in changes.items():
            setattr(out, k, v)
        return out

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in _FIELDS}


def default_para(**changes):
    """The reference's LocalizationPara() defaults (bfgs_base.cu:18-86)."""
    p = LocPara()
    p.KAdc, p.Offset, p.QE, p.ReadNoise_e = 0.45, 100, 0.72, 1.3
    p.ROISize, p.LocType, p.MultiEmitterFitEn, p.WLEEn = 7, 0, 0, 1
    p.ConsecFit_DistanceTh_nm, p.ConsecFitEn = 80.0, 0
    p.PixelSize, p.PixelZoom, p.SNR_th, p.ColorMode_3D = 100, 5, 5, 0
    p.ImageWidth, p.ImageHigh, p.TotalFrameNum = 2048, 2048, 1
    p.MinZDepth, p.MaxZDepth, p.ZDepthCorrFactor = -500, 500, 1.0
    p.p4_XGY, p.p3_XGY, p.p2_XGY, p.p1_XGY, p.p0_XGY = 0, 0, 0, 1, 0
    p.p4_XLY, p.p3_XLY, p.p2_XLY, p.p1_XLY, p.p0_XLY = 0, 0, 0, 1, 0
    p.DH_RotateType, p.DH_MeanDistance, p.DH_DistanceTh = 0, 10.0, 2.0
    p.ImagesPerGroup, p.IsHollowTube, p.StrucuteSize_2D = 50, 0, 40
    p.SpatialResolutionCalcEn = 1
    p.SRImageWidth = (int(p.ImageWidth * p.PixelZoom) + 3) // 4 * 4
    p.SRImageHigh = (int(p.ImageHigh * p.PixelZoom) + 3) // 4 * 4
    for k, v in changes.items():
        setattr(p, k, v)
    return p


def ptr(a):
    """Data pointer of a numpy array (None for None)."""
    return None if a is None else C.c_void_p(a.ctypes.data)


PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(PKG_DIR), "lib", "libqcstorm_b200.so")
