/*
 * gdalIO/gdalIO/grimpgdal.h -- TEST INFRASTRUCTURE ONLY.  Type names of the
 * GDAL interface the reference's sources mention (GDAL is not installed).
 * The parity harness reads raw image files, so GDALRasterIO is never reached;
 * its stand-in fails loudly if it is.
 */
#ifndef REFSHIM_GRIMPGDAL_H
#define REFSHIM_GRIMPGDAL_H
typedef void *GDALRasterBandH;
typedef void *GDALDatasetH;
typedef enum { CE_None = 0, CE_Failure = 3 } CPLErr;
typedef enum { GDT_Unknown = 0, GDT_Byte = 1, GDT_Int16 = 3, GDT_Int32 = 5, GDT_Float32 = 6, GDT_CInt16 = 8,
               GDT_CFloat32 = 10 } GDALDataType;
typedef enum { GF_Read = 0, GF_Write = 1 } GDALRWFlag;
/* dictionary node of GrIMP's VRT metadata (only passed around) */
typedef struct dictNodeType dictNode;
CPLErr GDALRasterIO(GDALRasterBandH hBand, GDALRWFlag eRWFlag, int nXOff, int nYOff, int nXSize, int nYSize,
                    void *pData, int nBufXSize, int nBufYSize, GDALDataType eBufType, int nPixelSpace,
                    int nLineSpace);
#endif
