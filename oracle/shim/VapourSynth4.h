/* Oracle build shim (test infrastructure only).
 *
 * This is not the VapourSynth API header. The reference's compute translation
 * units name a few VapourSynth types in lgcr.h without using their members;
 * its Downsample translation unit (src/downsample.cpp) calls the API through
 * a function table. This file declares only the names those two need, with
 * the argument meaning of the VapourSynth v4 API, so the reference's own
 * Downsample code compiles unmodified against the oracle's in-memory host
 * (oracle/ds_host.cpp), which implements every entry below. Member order and
 * enumerator values are this shim's own: nothing built against it talks to
 * a real VapourSynth core. */
#pragma once

#include <cstddef>
#include <cstdint>

#define VS_CC

struct VSNode;
struct VSCore;
struct VSPlugin;
struct VSFrame;
struct VSMap;
struct VSFrameContext;
struct VSAPI;
struct VSPLUGINAPI;

enum VSColorFamily { cfUndefined = 0, cfGray = 1, cfRGB = 2, cfYUV = 3 };
enum VSSampleType { stInteger = 0, stFloat = 1 };
enum VSMapAppendMode { maReplace = 0, maAppend = 1 };
enum VSActivationReason { arInitial = 0, arAllFramesReady = 1, arError = -1 };
enum VSRequestPattern { rpGeneral = 0, rpNoFrameReuse = 1, rpStrictSpatial = 2 };
enum VSFilterMode { fmParallel = 0, fmParallelRequests = 1, fmUnordered = 2, fmFrameState = 3 };

struct VSVideoFormat {
    int colorFamily;
    int sampleType;
    int bitsPerSample;
    int bytesPerSample;
    int subSamplingW;
    int subSamplingH;
    int numPlanes;
};

struct VSVideoInfo {
    VSVideoFormat format;
    int64_t fpsNum;
    int64_t fpsDen;
    int width;
    int height;
    int numFrames;
};

struct VSFilterDependency {
    VSNode *source;
    int requestPattern;
};

typedef const VSFrame *(VS_CC *VSFilterGetFrame)(int n, int activationReason, void *instanceData,
                                                  void **frameData, VSFrameContext *frameCtx,
                                                  VSCore *core, const VSAPI *vsapi);
typedef void (VS_CC *VSFilterFree)(void *instanceData, VSCore *core, const VSAPI *vsapi);
typedef void (VS_CC *VSPublicFunction)(const VSMap *in, VSMap *out, void *userData,
                                       VSCore *core, const VSAPI *vsapi);

struct VSAPI {
    // filters and frames
    void (VS_CC *createVideoFilter)(VSMap *out, const char *name, const VSVideoInfo *vi,
                                    VSFilterGetFrame getFrame, VSFilterFree free,
                                    int filterMode, const VSFilterDependency *dependencies,
                                    int numDeps, void *instanceData, VSCore *core);
    const VSFrame *(VS_CC *getFrameFilter)(int n, VSNode *node, VSFrameContext *frameCtx);
    void (VS_CC *requestFrameFilter)(int n, VSNode *node, VSFrameContext *frameCtx);
    VSFrame *(VS_CC *newVideoFrame2)(const VSVideoFormat *format, int width, int height,
                                     const VSFrame **planeSrc, const int *planes,
                                     const VSFrame *propSrc, VSCore *core);
    void (VS_CC *freeFrame)(const VSFrame *f);
    void (VS_CC *freeNode)(VSNode *node);
    const VSVideoInfo *(VS_CC *getVideoInfo)(VSNode *node);
    const VSVideoFormat *(VS_CC *getVideoFrameFormat)(const VSFrame *f);
    const uint8_t *(VS_CC *getReadPtr)(const VSFrame *f, int plane);
    uint8_t *(VS_CC *getWritePtr)(VSFrame *f, int plane);
    ptrdiff_t (VS_CC *getStride)(const VSFrame *f, int plane);
    int (VS_CC *queryVideoFormat)(VSVideoFormat *format, int colorFamily, int sampleType,
                                  int bitsPerSample, int subSamplingW, int subSamplingH,
                                  VSCore *core);
    // property maps
    VSMap *(VS_CC *getFramePropertiesRW)(VSFrame *f);
    void (VS_CC *mapSetError)(VSMap *map, const char *errorMessage);
    VSNode *(VS_CC *mapGetNode)(const VSMap *map, const char *key, int index, int *error);
    int (VS_CC *mapGetIntSaturated)(const VSMap *map, const char *key, int index, int *error);
    float (VS_CC *mapGetFloatSaturated)(const VSMap *map, const char *key, int index, int *error);
    const char *(VS_CC *mapGetData)(const VSMap *map, const char *key, int index, int *error);
    int (VS_CC *mapSetInt)(VSMap *map, const char *key, int64_t i, int append);
    int (VS_CC *mapSetFloat)(VSMap *map, const char *key, double d, int append);
};

struct VSPLUGINAPI {
    int (VS_CC *registerFunction)(const char *name, const char *args, const char *returnType,
                                  VSPublicFunction argsFunc, void *functionData,
                                  VSPlugin *plugin);
};
