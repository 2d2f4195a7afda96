// Oracle in-memory host for the reference's Downsample filter (test
// infrastructure only: the parity checker, never a product path).
//
// The reference's Downsample (src/downsample.cpp) keeps all of its code in an
// anonymous namespace behind the VapourSynth API: registerDownsample
// (downsample.cpp:913-918) hands downsampleCreate to the plugin API, create
// (820-911) parses the argument map and registers downsampleGetFrame (740-781)
// with the core. This file implements the few API entries those functions
// call (declared by shim/VapourSynth4.h) over plain host memory and drives
// them the way a VapourSynth core does for one frame: register, create,
// request (arInitial), compute (arAllFramesReady), free. The reference's code
// runs unmodified; only the core around it is stood in for.
#include <VapourSynth4.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

namespace lgcr {
void registerDownsample(VSPlugin *plugin, const VSPLUGINAPI *vspapi);
}

struct VSCore { int unused; };
struct VSFrameContext { int unused; };

struct VSMap {
    VSNode *node = nullptr;
    std::map<std::string, int64_t> ints;
    std::map<std::string, double> floats;
    std::map<std::string, std::string> data;
    std::string error;
    // what createVideoFilter registered
    VSFilterGetFrame getFrame = nullptr;
    VSFilterFree freeFn = nullptr;
    void *instance = nullptr;
    VSVideoInfo vi{};
};

struct VSFrame {
    VSVideoFormat fmt{};
    int w[3] = {0, 0, 0}, h[3] = {0, 0, 0};
    const uint8_t *rd[3] = {nullptr, nullptr, nullptr};
    uint8_t *wr[3] = {nullptr, nullptr, nullptr};
    ptrdiff_t stride[3] = {0, 0, 0};
    std::vector<uint8_t> own[3];
    VSMap props;
    bool owned = false;                 // allocated by newVideoFrame2
};

struct VSNode {
    VSVideoInfo vi{};
    VSFrame *frame = nullptr;
};

namespace {

VSPublicFunction g_create = nullptr;

void VS_CC createVideoFilter(VSMap *out, const char *, const VSVideoInfo *vi, VSFilterGetFrame getFrame,
                             VSFilterFree freeFn, int, const VSFilterDependency *, int, void *instance,
                             VSCore *) {
    out->getFrame = getFrame;
    out->freeFn = freeFn;
    out->instance = instance;
    out->vi = *vi;
}

const VSFrame *VS_CC getFrameFilter(int, VSNode *node, VSFrameContext *) { return node->frame; }
void VS_CC requestFrameFilter(int, VSNode *, VSFrameContext *) {}

VSFrame *VS_CC newVideoFrame2(const VSVideoFormat *format, int width, int height, const VSFrame **planeSrc,
                              const int *planes, const VSFrame *propSrc, VSCore *) {
    auto *f = new VSFrame;
    f->fmt = *format;
    f->owned = true;
    for (int p = 0; p < format->numPlanes && p < 3; ++p) {
        const int pw = p ? width >> format->subSamplingW : width;
        const int ph = p ? height >> format->subSamplingH : height;
        f->w[p] = pw;
        f->h[p] = ph;
        if (planeSrc && planeSrc[p]) {
            // shared plane: read-only view of the source frame's plane
            const VSFrame *s = planeSrc[p];
            f->rd[p] = s->rd[planes[p]];
            f->stride[p] = s->stride[planes[p]];
        } else {
            f->stride[p] = ptrdiff_t(pw) * format->bytesPerSample;
            f->own[p].assign(size_t(f->stride[p]) * ph, 0);
            f->wr[p] = f->own[p].data();
            f->rd[p] = f->wr[p];
        }
    }
    if (propSrc) {
        f->props.ints = propSrc->props.ints;
        f->props.floats = propSrc->props.floats;
        f->props.data = propSrc->props.data;
    }
    return f;
}

void VS_CC freeFrame(const VSFrame *f) {
    if (f && f->owned)
        delete f;
}
void VS_CC freeNode(VSNode *) {}
const VSVideoInfo *VS_CC getVideoInfo(VSNode *node) { return &node->vi; }
const VSVideoFormat *VS_CC getVideoFrameFormat(const VSFrame *f) { return &f->fmt; }
const uint8_t *VS_CC getReadPtr(const VSFrame *f, int p) { return f->rd[p]; }
uint8_t *VS_CC getWritePtr(VSFrame *f, int p) { return f->wr[p]; }
ptrdiff_t VS_CC getStride(const VSFrame *f, int p) { return f->stride[p]; }

int VS_CC queryVideoFormat(VSVideoFormat *format, int colorFamily, int sampleType, int bitsPerSample,
                           int subSamplingW, int subSamplingH, VSCore *) {
    format->colorFamily = colorFamily;
    format->sampleType = sampleType;
    format->bitsPerSample = bitsPerSample;
    format->bytesPerSample = bitsPerSample <= 8 ? 1 : bitsPerSample <= 16 ? 2 : 4;
    format->subSamplingW = subSamplingW;
    format->subSamplingH = subSamplingH;
    format->numPlanes = colorFamily == cfGray ? 1 : 3;
    return 1;
}

VSMap *VS_CC getFramePropertiesRW(VSFrame *f) { return &f->props; }
void VS_CC mapSetError(VSMap *map, const char *msg) { map->error = msg; }

VSNode *VS_CC mapGetNode(const VSMap *map, const char *key, int, int *error) {
    const bool ok = std::strcmp(key, "clip") == 0 && map->node;
    if (error)
        *error = ok ? 0 : 1;
    return ok ? map->node : nullptr;
}

int VS_CC mapGetIntSaturated(const VSMap *map, const char *key, int, int *error) {
    auto it = map->ints.find(key);
    if (error)
        *error = it == map->ints.end();
    if (it == map->ints.end())
        return 0;
    return int(std::max<int64_t>(INT_MIN, std::min<int64_t>(INT_MAX, it->second)));
}

float VS_CC mapGetFloatSaturated(const VSMap *map, const char *key, int, int *error) {
    auto it = map->floats.find(key);
    if (error)
        *error = it == map->floats.end();
    return it == map->floats.end() ? 0.0f : float(it->second);
}

const char *VS_CC mapGetData(const VSMap *map, const char *key, int, int *error) {
    auto it = map->data.find(key);
    if (error)
        *error = it == map->data.end();
    return it == map->data.end() ? nullptr : it->second.c_str();
}

int VS_CC mapSetInt(VSMap *map, const char *key, int64_t i, int) {
    map->ints[key] = i;
    return 0;
}

int VS_CC mapSetFloat(VSMap *map, const char *key, double d, int) {
    map->floats[key] = d;
    return 0;
}

int VS_CC registerFunction(const char *name, const char *, const char *, VSPublicFunction fn, void *,
                           VSPlugin *) {
    if (std::strcmp(name, "Downsample") == 0)
        g_create = fn;
    return 1;
}

const VSAPI g_api = {
    createVideoFilter, getFrameFilter, requestFrameFilter, newVideoFrame2, freeFrame, freeNode,
    getVideoInfo, getVideoFrameFormat, getReadPtr, getWritePtr, getStride, queryVideoFormat,
    getFramePropertiesRW, mapSetError, mapGetNode, mapGetIntSaturated, mapGetFloatSaturated,
    mapGetData, mapSetInt, mapSetFloat,
};

const VSPLUGINAPI g_pluginApi = { registerFunction };

void copyError(const std::string &msg, char *err, int errlen) {
    if (err && errlen > 0) {
        std::strncpy(err, msg.c_str(), size_t(errlen) - 1);
        err[errlen - 1] = '\0';
    }
}

} // namespace

extern "C" {

// One Downsample frame through the reference's own create / getFrame.
//   format: color_family (3 = YUV), sample_type (0 int, 1 float), bits,
//           subsampling; planes / strides describe the source frame (planes
//           may be null to check only the create-time validation)
//   arguments: quality (INT_MIN = not given), kernel / loc (null = not
//           given), strength (used when strength_given is nonzero)
//   out_u / out_v: (width >> 1) x (height >> 1) packed samples
// Returns 0, or 1 with the reference's error message in err.
int oracle_downsample_frame(int width, int height, int color_family, int sample_type, int bits,
                            int ssw, int ssh, const void *const planes[3], const long long strides[3],
                            int quality, const char *kernel, double strength, int strength_given,
                            const char *loc,
                            void *out_u, void *out_v, int *chroma_location, char *err, int errlen) {
    static std::once_flag once;
    std::call_once(once, [] { lgcr::registerDownsample(nullptr, &g_pluginApi); });
    if (!g_create) {
        copyError("oracle: Downsample was not registered", err, errlen);
        return 1;
    }
    VSCore core{};
    VSFrameContext ctx{};
    VSNode node;
    queryVideoFormat(&node.vi.format, color_family, sample_type, bits, ssw, ssh, &core);
    node.vi.width = width;
    node.vi.height = height;
    node.vi.numFrames = 1;
    VSFrame src;
    src.fmt = node.vi.format;
    for (int p = 0; p < 3; ++p) {
        src.w[p] = p ? width >> ssw : width;
        src.h[p] = p ? height >> ssh : height;
        src.rd[p] = planes ? static_cast<const uint8_t *>(planes[p]) : nullptr;
        src.stride[p] = strides ? ptrdiff_t(strides[p]) : 0;
    }
    node.frame = &src;

    VSMap in, out;
    in.node = &node;
    if (quality != INT_MIN)
        in.ints["quality"] = quality;
    if (kernel)
        in.data["kernel"] = kernel;
    if (strength_given)
        in.floats["strength"] = strength;
    if (loc)
        in.data["loc"] = loc;
    g_create(&in, &out, nullptr, &core, &g_api);
    if (!out.error.empty()) {
        copyError(out.error, err, errlen);
        return 1;
    }
    if (!out.getFrame) {
        copyError("oracle: Downsample did not create a filter", err, errlen);
        return 1;
    }
    int rc = 0;
    if (planes) {
        void *frameData = nullptr;
        out.getFrame(0, arInitial, out.instance, &frameData, &ctx, &core, &g_api);
        const VSFrame *dst = out.getFrame(0, arAllFramesReady, out.instance, &frameData, &ctx, &core, &g_api);
        if (!dst) {
            copyError("oracle: Downsample returned no frame", err, errlen);
            rc = 1;
        } else {
            const int bps = dst->fmt.bytesPerSample;
            void *outs[2] = {out_u, out_v};
            for (int p = 1; p < 3; ++p)
                for (int y = 0; y < dst->h[p]; ++y)
                    std::memcpy(static_cast<uint8_t *>(outs[p - 1]) + size_t(y) * dst->w[p] * bps,
                                dst->rd[p] + ptrdiff_t(y) * dst->stride[p], size_t(dst->w[p]) * bps);
            auto it = dst->props.ints.find("_ChromaLocation");
            if (chroma_location)
                *chroma_location = it == dst->props.ints.end() ? -1 : int(it->second);
            freeFrame(dst);
        }
    }
    if (out.freeFn)
        out.freeFn(out.instance, &core, &g_api);
    return rc;
}

} // extern "C"
