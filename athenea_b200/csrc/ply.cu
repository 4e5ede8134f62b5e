// The 3DGS PLY reader: a trained splat cloud's vertex element as float
// records and the encoding that names their fields, ready for
// ath_decode_records. Host code only.
//
// It reads what the reference's readSplatPly reads (modules/io/src/SplatReaders.cpp:50-200,
// header grammar modules/io/src/PlyHeader.cpp): binary little-endian files only;
// a vertex element with no list property; x y z, opacity, scale_0..2, rot_0..3
// (w x y z) and f_dc_0..2 required; the f_rest_* harmonics counted, contiguous
// and colour-outermost, a whole degree (9, 24 or 45 of them; fewer than 9 are
// ignored, as the reference ignores them); every property
// widened to one float of the record, in the file's order; elements before the
// vertex element skipped by their size. The errors are the reference's: a bad
// header or missing property is InvalidArgument, another format, a list, a
// property type it does not know or harmonics that are not a whole degree are
// Unsupported, a file that ends early is IoFailure.
#include <cstdint>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/athenea_raster.h"
#include "host_util.h"

using namespace ath;

namespace {

struct PlyProperty {
    std::string name, type;
    uint32_t offset = 0, size = 0;
    bool list = false;
};

struct PlyElement {
    std::string name;
    uint64_t count = 0;
    uint32_t stride = 0;
    bool hasList = false;
    std::vector<PlyProperty> properties;

    int find(const std::string& n) const {
        for (size_t k = 0; k < properties.size(); ++k)
            if (properties[k].name == n) return (int)k;
        return -1;
    }
};

uint32_t sizeOfType(const std::string& t) {
    if (t == "char" || t == "uchar" || t == "int8" || t == "uint8") return 1;
    if (t == "short" || t == "ushort" || t == "int16" || t == "uint16") return 2;
    if (t == "int" || t == "uint" || t == "int32" || t == "uint32" || t == "float" || t == "float32") return 4;
    if (t == "double" || t == "float64") return 8;
    return 0;
}

double valueAt(const unsigned char* at, const std::string& t) {
    if (t == "float" || t == "float32") { float v; std::memcpy(&v, at, 4); return v; }
    if (t == "double" || t == "float64") { double v; std::memcpy(&v, at, 8); return v; }
    if (t == "uchar" || t == "uint8") return *at;
    if (t == "char" || t == "int8") return (int8_t)*at;
    if (t == "ushort" || t == "uint16") { uint16_t v; std::memcpy(&v, at, 2); return v; }
    if (t == "short" || t == "int16") { int16_t v; std::memcpy(&v, at, 2); return v; }
    if (t == "uint" || t == "uint32") { uint32_t v; std::memcpy(&v, at, 4); return v; }
    int32_t v;
    std::memcpy(&v, at, 4);
    return v;
}

struct Cloud {
    std::string format;
    std::vector<PlyElement> elements;
    size_t dataStart = 0;      // bytes: where the first element's data begins
    const PlyElement* vertex = nullptr;
    size_t vertexStart = 0;    // bytes: where the vertex element's data begins
    ath_encoding encoding{};
};

ath_status fromHeader(const std::string& path, std::ifstream& in, Cloud& c) {
    std::string line;
    if (!std::getline(in, line) || line.rfind("ply", 0) != 0)
        return fail(ATH_E_INVALID_ARGUMENT, "'" + path + "': not a PLY file");
    bool ended = false;
    while (std::getline(in, line)) {
        if (!line.empty() && line.back() == '\r') line.pop_back();
        std::istringstream words(line);
        std::string word;
        words >> word;
        if (word == "format") {
            words >> c.format;
        } else if (word == "element") {
            PlyElement e;
            words >> e.name >> e.count;
            c.elements.push_back(e);
        } else if (word == "property") {
            if (c.elements.empty()) return fail(ATH_E_INVALID_ARGUMENT, "'" + path + "': a PLY property before any element");
            PlyElement& e = c.elements.back();
            PlyProperty p;
            std::string type;
            words >> type;
            if (type == "list") {
                std::string countType, itemType;
                words >> countType >> itemType >> p.name;
                p.type = "list";
                p.list = true;
                e.hasList = true;
            } else {
                words >> p.name;
                p.type = type;
                p.offset = e.stride;
                p.size = sizeOfType(type);
                e.stride += p.size;
            }
            e.properties.push_back(p);
        } else if (word == "end_header") {
            ended = true;
            break;
        }
    }
    if (!ended) return fail(ATH_E_INVALID_ARGUMENT, "'" + path + "': the PLY header has no end_header");
    c.dataStart = (size_t)in.tellg();
    if (c.format != "binary_little_endian")
        return fail(ATH_E_UNSUPPORTED, "'" + path + "': PLY format '" + c.format + "'; splat clouds are binary_little_endian");
    size_t offset = c.dataStart;
    for (const PlyElement& e : c.elements) {
        if (e.name == "vertex") {
            c.vertex = &e;
            c.vertexStart = offset;
            break;
        }
        if (e.hasList)
            return fail(ATH_E_UNSUPPORTED, "'" + path + "': a list element ('" + e.name +
                                               "') before 'vertex' makes its offset unknowable");
        offset += (size_t)e.stride * e.count;
    }
    if (!c.vertex || c.vertex->count == 0) return fail(ATH_E_INVALID_ARGUMENT, "'" + path + "': no vertices");
    const PlyElement& v = *c.vertex;
    if (v.hasList) return fail(ATH_E_UNSUPPORTED, "'" + path + "': a list in the vertex element");
    if (v.count > 0xFFFFFFFFull) return fail(ATH_E_UNSUPPORTED, "'" + path + "': more than 2^32 splats");
    for (const PlyProperty& p : v.properties)
        if (p.size == 0)
            return fail(ATH_E_UNSUPPORTED, "'" + path + "': property '" + p.name + "' of type '" + p.type + "'");
    static const char* kRequired[] = {"x", "y", "z", "opacity", "scale_0", "scale_1", "scale_2",
                                      "rot_0", "rot_1", "rot_2", "rot_3", "f_dc_0", "f_dc_1", "f_dc_2"};
    for (const char* n : kRequired)
        if (v.find(n) < 0)
            return fail(ATH_E_INVALID_ARGUMENT,
                        "'" + path + "': no '" + n + "' -- this does not look like a trained splat cloud");
    ath_encoding& e = c.encoding;
    e.stride = (uint32_t)v.properties.size();
    e.x = v.find("x"); e.y = v.find("y"); e.z = v.find("z");
    e.opacity = v.find("opacity");
    e.scale0 = v.find("scale_0"); e.scale1 = v.find("scale_1"); e.scale2 = v.find("scale_2");
    e.rot_w = v.find("rot_0"); e.rot_x = v.find("rot_1"); e.rot_y = v.find("rot_2"); e.rot_z = v.find("rot_3");
    e.dc0 = v.find("f_dc_0"); e.dc1 = v.find("f_dc_1"); e.dc2 = v.find("f_dc_2");
    uint32_t restCount = 0;
    for (const PlyProperty& p : v.properties)
        if (p.name.rfind("f_rest_", 0) == 0) ++restCount;
    uint32_t perColour = 0;
    for (uint32_t basis : {15u, 8u, 3u})
        if (restCount >= basis * 3) {
            perColour = basis;
            break;
        }
    e.rest_base = 0;
    e.file_per_colour = 0;
    e.keep_per_colour = perColour;
    if (perColour > 0) {
        if (restCount / 3 != perColour || restCount % 3 != 0)
            return fail(ATH_E_UNSUPPORTED,
                        "'" + path + "': " + std::to_string(restCount) + " harmonic coefficients is not a whole degree");
        e.rest_base = v.find("f_rest_0");
        e.file_per_colour = perColour;
        for (uint32_t k = 0; k < perColour * 3; ++k) {
            const std::string n = "f_rest_" + std::to_string(k);
            if (v.find(n) != (int)(e.rest_base + k))
                return fail(ATH_E_UNSUPPORTED, "'" + path + "': harmonics are not contiguous in the vertex element");
        }
    }
    return ATH_OK;
}

ath_status openCloud(const char* path, std::ifstream& in, Cloud& c) {
    if (!path) return fail(ATH_E_INVALID_ARGUMENT, "ath_ply_read: null path");
    in.open(path, std::ios::binary);
    if (!in) return fail(ATH_E_NOT_FOUND, std::string("'") + path + "': cannot open");
    return fromHeader(path, in, c);
}

}   // namespace

extern "C" ath_status ath_ply_read_header(const char* path, uint32_t* count, ath_encoding* encoding) {
    std::ifstream in;
    Cloud c;
    ath_status st = openCloud(path, in, c);
    if (st != ATH_OK) return st;
    if (count) *count = (uint32_t)c.vertex->count;
    if (encoding) *encoding = c.encoding;
    return ATH_OK;
}

extern "C" ath_status ath_ply_read(const char* path, float* records, uint64_t capacity, uint32_t* count,
                                   ath_encoding* encoding) {
    std::ifstream in;
    Cloud c;
    ath_status st = openCloud(path, in, c);
    if (st != ATH_OK) return st;
    const PlyElement& v = *c.vertex;
    const uint64_t floats = (uint64_t)v.count * c.encoding.stride;
    if (!records || capacity < floats)
        return fail(ATH_E_INVALID_ARGUMENT, "ath_ply_read: room for " + std::to_string(floats) + " floats needed");
    in.seekg(0, std::ios::end);
    const size_t size = (size_t)in.tellg();
    if (c.vertexStart + (size_t)v.stride * v.count > size)
        return fail(ATH_E_IO_FAILURE, std::string("'") + path + "': the file ends before its vertices do");
    in.seekg((std::streamoff)c.vertexStart);
    std::vector<unsigned char> block((size_t)v.stride * 4096);
    for (uint64_t first = 0; first < v.count; first += 4096) {
        const uint64_t n = std::min<uint64_t>(4096, v.count - first);
        if (!in.read(reinterpret_cast<char*>(block.data()), (std::streamsize)(n * v.stride)))
            return fail(ATH_E_IO_FAILURE, std::string("'") + path + "': a read failed");
        for (uint64_t i = 0; i < n; ++i) {
            const unsigned char* rec = block.data() + i * v.stride;
            float* out = records + (first + i) * c.encoding.stride;
            for (size_t k = 0; k < v.properties.size(); ++k)
                out[k] = (float)valueAt(rec + v.properties[k].offset, v.properties[k].type);
        }
    }
    if (count) *count = (uint32_t)v.count;
    if (encoding) *encoding = c.encoding;
    return ATH_OK;
}
