// NIfTI-1 reader (io/nifti.rs read / read_info), for 3-D scalar volumes, so the metric
// can be fed from the format most registration data comes in.
//
// Files: a single `.nii` (magic "n+1"), a `.hdr` + `.img` pair (magic "ni1"), or an
// Analyze-7.5 pair (no magic), each optionally gzip-compressed (`.nii.gz`, `.hdr.gz`,
// `.img.gz`: a name ending in .gz is read through zlib, which also passes plain bytes
// through; any other name is read raw). The header's byte order follows dim[0], or
// sizeof_hdr when dim[0] is 0 (nifti.rs need_nhdr_swap, :822-842).
//
// Geometry follows NiftiImageIO's read path as the reference restates it:
// - the quaternion form (qform_code > 0, NIfTI only) gives qto_xyz, else the diagonal
//   of pixdim; the sform (sform_code > 0) gives sto_xyz, else zeros (nifti.rs:1150-1200);
// - the matrix used is chosen by the_mat (nifti.rs:1724-1768): the sform when the two
//   agree, or when the sform is an invertible affine without skew and either the
//   qform is unknown, the sform is scanner-anatomical, or an SVD comparison finds the
//   two very similar; its polar factor under ITK_NIFTI_SFORM_PERMISSIVE when it has
//   skew; else the qform when known; else the read is refused;
// - NIfTI is RAS+, the library LPS: origin (−m03, −m13, m23) and direction columns
//   (−m0d, −m1d, m2d) normalised (nifti.rs:1795-1876); both codes unknown gives origin 0
//   and the identity;
// - spacing is pixdim[1..3] in millimetres (xyz_units metres ×1000, microns ×1e-3).
// Intensity: scl_slope / scl_inter (not for Analyze; a slope below DBL_EPSILON is 1)
// rescale every voxel, integer types first cast to f32 and the result stored as f32
// (nifti.rs:2085-2099, :2254-2300).
// Refused by name: dimensions other than 3 once trailing unit dimensions are dropped,
// vector / matrix intents, complex and RGB datatypes (MI_ERR_UNSUPPORTED_PIXEL_TYPE),
// unknown datatypes, truncated data.
#include <zlib.h>

#include <cctype>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iterator>
#include <string>
#include <sys/stat.h>
#include <type_traits>
#include <vector>

#include "internal.h"

namespace mi {
namespace {

constexpr int HDR = 348;
constexpr int16_t DT_UINT8 = 2, DT_INT16 = 4, DT_INT32 = 8, DT_FLOAT32 = 16, DT_COMPLEX64 = 32, DT_FLOAT64 = 64,
                  DT_RGB24 = 128, DT_INT8 = 256, DT_UINT16 = 512, DT_UINT32 = 768, DT_INT64 = 1024,
                  DT_UINT64 = 1280, DT_COMPLEX128 = 1792, DT_RGBA32 = 2304;
constexpr int16_t INTENT_GENMATRIX = 1004, INTENT_SYMMATRIX = 1005, INTENT_DISPVECT = 1006, INTENT_VECTOR = 1007;
constexpr int16_t XFORM_UNKNOWN = 0, XFORM_SCANNER_ANAT = 1;
constexpr int FTYPE_ANALYZE = 0, FTYPE_NIFTI1_1 = 1, FTYPE_NIFTI1_2 = 2;

using M44 = float[4][4];
using M33 = float[3][3];

struct Fail {
    mi_status s;
    std::string why;
};

// ---- file names (nifti.rs:1313-1560: nifti_find_file_extension and friends) ----

bool has_lower(const std::string& s) {
    for (char c : s)
        if (std::islower((unsigned char)c)) return true;
    return false;
}
bool has_upper(const std::string& s) {
    for (char c : s)
        if (std::isupper((unsigned char)c)) return true;
    return false;
}
std::string lower(std::string s) {
    for (auto& c : s) c = (char)std::tolower((unsigned char)c);
    return s;
}
std::string upper(std::string s) {
    for (auto& c : s) c = (char)std::toupper((unsigned char)c);
    return s;
}

// The recognised extension at the end of name ("" when none): .nii .hdr .img .nia,
// or .nii.gz .hdr.gz .img.gz; mixed case is not an extension.
std::string file_extension(const std::string& name) {
    if (name.size() < 4) return "";
    std::string e = name.substr(name.size() - 4);
    const std::string le = lower(e);
    if (le == ".nii" || le == ".hdr" || le == ".img" || le == ".nia") return has_lower(e) && has_upper(e) ? "" : e;
    if (name.size() < 7) return "";
    e = name.substr(name.size() - 7);
    const std::string le7 = lower(e);
    if (le7 == ".nii.gz" || le7 == ".hdr.gz" || le7 == ".img.gz") return has_lower(e) && has_upper(e) ? "" : e;
    return "";
}

bool exists(const std::string& p) {
    struct stat st;
    return ::stat(p.c_str(), &st) == 0;
}

bool is_upper_ext(const std::string& e) { return !e.empty() && !has_lower(e) && has_upper(e); }
std::string cased(const std::string& s, bool up) { return up ? upper(s) : s; }

// nifti_findhdrname (nifti.rs:1468-1513)
bool find_hdr_name(const std::string& name, std::string& out) {
    const std::string ext = file_extension(name);
    if (name.empty() || ext.size() == name.size()) return false;
    const std::string base = name.substr(0, name.size() - ext.size());
    const bool up = is_upper_ext(ext);
    bool hdr_first = false;
    if (!ext.empty() && exists(name)) {
        if (lower(ext.substr(0, 4)) != ".img") {
            out = name;
            return true;
        }
        hdr_first = true;
    }
    const char* order[2] = {hdr_first ? ".hdr" : ".nii", hdr_first ? ".nii" : ".hdr"};
    for (const char* stem : order)
        for (const char* gz : {"", ".gz"}) {
            const std::string c = base + cased(stem, up) + cased(gz, up);
            if (exists(c)) {
                out = c;
                return true;
            }
        }
    return false;
}

// nifti_makeimgname on the found header name (nifti.rs:1422-1462)
std::string make_img_name(const std::string& prefix, bool comp) {
    std::string iname = prefix;
    const std::string ext = file_extension(iname);
    const bool up = is_upper_ext(ext);
    if (!ext.empty()) {
        if (ext.substr(0, 4) == cased(".hdr", up)) iname.replace(iname.size() - ext.size(), 4, cased(".img", up));
        if (comp && iname.find(cased(".gz", up)) == std::string::npos) iname += cased(".gz", up);
    } else {
        iname += ".img";
        if (comp) iname += ".gz";
    }
    return iname;
}

// nifti_findimgname (nifti.rs:1515-1544)
bool find_img_name(const std::string& iname, int ftype, std::string& out) {
    const std::string ext = file_extension(iname);
    if (iname.empty() || ext.size() == iname.size()) return false;
    const std::string base = iname.substr(0, iname.size() - ext.size());
    const bool up = is_upper_ext(ext);
    const char* order[2] = {ftype == FTYPE_NIFTI1_1 ? ".nii" : ".img", ftype == FTYPE_NIFTI1_1 ? ".img" : ".nii"};
    for (const char* stem : order)
        for (const char* gz : {"", ".gz"}) {
            const std::string c = base + cased(stem, up) + cased(gz, up);
            if (exists(c)) {
                out = c;
                return true;
            }
        }
    return false;
}

bool is_gz(const std::string& p) { return p.size() >= 3 && lower(p.substr(p.size() - 3)) == ".gz"; }

// The whole file: through zlib when the name ends in .gz (zlib passes plain bytes
// through), raw otherwise. `limit` > 0 stops after that many bytes.
bool read_bytes(const std::string& path, std::string& out, size_t limit = 0) {
    out.clear();
    if (is_gz(path)) {
        gzFile f = gzopen(path.c_str(), "rb");
        if (!f) return false;
        char buf[1 << 16];
        for (;;) {
            const size_t want = limit ? std::min(sizeof(buf), limit - out.size()) : sizeof(buf);
            if (want == 0) break;
            const int n = gzread(f, buf, (unsigned)want);
            if (n < 0) {
                gzclose(f);
                return false;
            }
            if (n == 0) break;
            out.append(buf, (size_t)n);
        }
        gzclose(f);
        return true;
    }
    std::ifstream f(path, std::ios::binary);
    if (!f) return false;
    if (limit) {
        out.resize(limit);
        f.read(&out[0], (std::streamsize)limit);
        out.resize((size_t)f.gcount());
    } else {
        out.assign(std::istreambuf_iterator<char>(f), std::istreambuf_iterator<char>());
    }
    return true;
}

// ---- the header (nifti.rs:773-980) ----

struct Header {
    int16_t dim[8];
    float pixdim[8];
    int16_t intent_code, datatype;
    float vox_offset, scl_slope, scl_inter;
    uint8_t xyzt_units;
    int16_t qform_code, sform_code;
    float qb, qc, qd, qx, qy, qz;
    float srow[3][4];
    char magic[4];
};

int16_t rd16(const unsigned char* b, int off, bool swap) {
    const uint16_t v = swap ? (uint16_t)((b[off] << 8) | b[off + 1]) : (uint16_t)(b[off] | (b[off + 1] << 8));
    return (int16_t)v;
}
uint32_t rd32u(const unsigned char* b, int off, bool swap) {
    uint32_t v = 0;
    for (int i = 0; i < 4; ++i) v |= (uint32_t)b[off + (swap ? 3 - i : i)] << (8 * i);
    return v;
}
float rdf(const unsigned char* b, int off, bool swap) {
    const uint32_t u = rd32u(b, off, swap);
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}
int16_t bswap16(int16_t v) { return (int16_t)(((uint16_t)v >> 8) | ((uint16_t)v << 8)); }
int32_t bswap32(int32_t v) {
    const uint32_t u = (uint32_t)v;
    return (int32_t)((u >> 24) | ((u >> 8) & 0xff00u) | ((u << 8) & 0xff0000u) | (u << 24));
}

bool parse_header(const std::string& bytes, Header& h, bool& swap, std::string& why) {
    if (bytes.size() < (size_t)HDR) {
        why = "the header is " + std::to_string(bytes.size()) + " bytes, need 348";
        return false;
    }
    const unsigned char* b = reinterpret_cast<const unsigned char*>(bytes.data());
    const int16_t dim0 = (int16_t)(b[40] | (b[41] << 8));
    int32_t hsize;
    std::memcpy(&hsize, b, 4);  // little-endian host
    if (dim0 != 0) {
        if (dim0 >= 1 && dim0 <= 7)
            swap = false;
        else if (bswap16(dim0) >= 1 && bswap16(dim0) <= 7)
            swap = true;
        else {
            why = "bad dim[0]";
            return false;
        }
    } else if (hsize == HDR) {
        swap = false;
    } else if (bswap32(hsize) == HDR) {
        swap = true;
    } else {
        why = "bad sizeof_hdr";
        return false;
    }
    for (int i = 0; i < 8; ++i) h.dim[i] = rd16(b, 40 + 2 * i, swap);
    for (int i = 0; i < 8; ++i) h.pixdim[i] = rdf(b, 76 + 4 * i, swap);
    h.intent_code = rd16(b, 68, swap);
    h.datatype = rd16(b, 70, swap);
    h.vox_offset = rdf(b, 108, swap);
    h.scl_slope = rdf(b, 112, swap);
    h.scl_inter = rdf(b, 116, swap);
    h.xyzt_units = b[123];
    h.qform_code = rd16(b, 252, swap);
    h.sform_code = rd16(b, 254, swap);
    h.qb = rdf(b, 256, swap);
    h.qc = rdf(b, 260, swap);
    h.qd = rdf(b, 264, swap);
    h.qx = rdf(b, 268, swap);
    h.qy = rdf(b, 272, swap);
    h.qz = rdf(b, 276, swap);
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 4; ++c) h.srow[r][c] = rdf(b, 280 + 16 * r + 4 * c, swap);
    std::memcpy(h.magic, b + 344, 4);
    return true;
}

// NIFTI_VERSION (nifti.rs:802-814): the version digit, 0 for an Analyze header
int nifti_version(const char* m) {
    if (m[0] == 'n' && m[3] == 0 && (m[1] == 'i' || m[1] == '+') && m[2] >= '1' && m[2] <= '9') return m[2] - '0';
    return 0;
}

float fixed_f32(float x) { return std::isfinite(x) ? x : 0.0f; }

// ---- small matrices (nifti.rs:209-700) ----

// nifti_quatern_to_mat44 (nifti.rs:377-437)
void quatern_to_mat44(float qb, float qc, float qd, float qx, float qy, float qz, float dx, float dy, float dz,
                      float qfac, M44 r) {
    double b = qb, c = qc, d = qd;
    double a = 1.0 - (b * b + c * c + d * d);
    if (a < 1.0e-7) {
        a = 1.0 / std::sqrt(b * b + c * c + d * d);
        b *= a;
        c *= a;
        d *= a;
        a = 0.0;
    } else {
        a = std::sqrt(a);
    }
    const double xd = dx > 0.0f ? (double)dx : 1.0, yd = dy > 0.0f ? (double)dy : 1.0;
    double zd = dz > 0.0f ? (double)dz : 1.0;
    if (qfac < 0.0f) zd = -zd;
    std::memset(r, 0, sizeof(M44));
    r[0][0] = (float)((a * a + b * b - c * c - d * d) * xd);
    r[0][1] = (float)(2.0 * (b * c - a * d) * yd);
    r[0][2] = (float)(2.0 * (b * d + a * c) * zd);
    r[1][0] = (float)(2.0 * (b * c + a * d) * xd);
    r[1][1] = (float)((a * a + c * c - b * b - d * d) * yd);
    r[1][2] = (float)(2.0 * (c * d - a * b) * zd);
    r[2][0] = (float)(2.0 * (b * d - a * c) * xd);
    r[2][1] = (float)(2.0 * (c * d + a * b) * yd);
    r[2][2] = (float)((a * a + d * d - c * c - b * b) * zd);
    r[0][3] = qx;
    r[1][3] = qy;
    r[2][3] = qz;
    r[3][3] = 1.0f;
}

// One-sided (Hestenes) Jacobi SVD of an N×N matrix: a = U·diag(w)·Vᵀ, w descending and
// non-negative, U's columns normalised (nifti.rs:549-638 states the same conventions).
template <int N>
void jacobi_svd(const double (&a)[N][N], double (&u)[N][N], double (&w)[N], double (&v)[N][N]) {
    for (int i = 0; i < N; ++i)
        for (int j = 0; j < N; ++j) {
            u[i][j] = a[i][j];
            v[i][j] = i == j ? 1.0 : 0.0;
        }
    for (int sweep = 0; sweep < 60; ++sweep) {
        bool converged = true;
        for (int p = 0; p < N - 1; ++p)
            for (int q = p + 1; q < N; ++q) {
                double alpha = 0.0, beta = 0.0, gamma = 0.0;
                for (int i = 0; i < N; ++i) {
                    alpha += u[i][p] * u[i][p];
                    beta += u[i][q] * u[i][q];
                    gamma += u[i][p] * u[i][q];
                }
                const double scale = std::sqrt(alpha * beta);
                if (gamma == 0.0 || std::fabs(gamma) <= 1e-300 * scale) continue;
                if (std::fabs(gamma) > DBL_EPSILON * scale) converged = false;
                const double zeta = (beta - alpha) / (2.0 * gamma);
                const double t = (zeta >= 0.0 ? 1.0 : -1.0) / (std::fabs(zeta) + std::sqrt(1.0 + zeta * zeta));
                const double c = 1.0 / std::sqrt(1.0 + t * t), s = c * t;
                for (int i = 0; i < N; ++i) {
                    const double up = u[i][p], uq = u[i][q];
                    u[i][p] = c * up - s * uq;
                    u[i][q] = s * up + c * uq;
                    const double vp = v[i][p], vq = v[i][q];
                    v[i][p] = c * vp - s * vq;
                    v[i][q] = s * vp + c * vq;
                }
            }
        if (converged) break;
    }
    for (int j = 0; j < N; ++j) {
        double n = 0.0;
        for (int i = 0; i < N; ++i) n += u[i][j] * u[i][j];
        w[j] = std::sqrt(n);
        if (w[j] > 0.0)
            for (int i = 0; i < N; ++i) u[i][j] /= w[j];
    }
    for (int i = 0; i < N; ++i) {
        int best = i;
        for (int j = i + 1; j < N; ++j)
            if (w[j] > w[best]) best = j;
        if (best != i) {
            std::swap(w[i], w[best]);
            for (int r = 0; r < N; ++r) {
                std::swap(u[r][i], u[r][best]);
                std::swap(v[r][i], v[r][best]);
            }
        }
    }
}

void top33(const M44 m, double (&o)[3][3]) {
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) o[i][j] = m[i][j];
}

template <int N>
bool is_identity(const float (&m)[N][N], double tol) {
    for (int i = 0; i < N; ++i)
        for (int j = 0; j < N; ++j) {
            const float dev = i == j ? std::fabs(m[i][j] - 1.0f) : std::fabs(m[i][j]);
            if ((double)dev > tol) return false;
        }
    return true;
}

// IsAffine (nifti.rs:649-669): bottom row (0,0,0,1) within float epsilon and an SVD
// condition number above double epsilon
bool is_affine(const M44 m) {
    double a[4][4];
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) a[i][j] = m[i][j];
    double err = std::fabs(a[3][3] - 1.0);
    for (int j = 0; j < 3; ++j) err += std::fabs(a[3][j]);
    if (err > (double)FLT_EPSILON) return false;
    double u[4][4], w[4], v[4][4];
    jacobi_svd<4>(a, u, w, v);
    return w[3] / w[0] > DBL_EPSILON;
}

// qform_sform_are_similar (nifti.rs:1660-1678)
bool qform_sform_similar(const M44 s, const M44 q) {
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            if ((double)std::fabs(s[i][j] - q[i][j]) > 1e-5) return false;
    double col = 0.0, row = 0.0;
    for (int i = 0; i < 4; ++i) col += std::fabs(s[i][3] - q[i][3]);
    if (col > 1e-7) return false;
    for (int j = 0; j < 4; ++j) row += std::fabs(s[3][j] - q[3][j]);
    return row <= 1e-7;
}

// sform_decomposable_without_skew (nifti.rs:1681-1700)
bool sform_without_skew(const M44 s) {
    if (!is_affine(s)) return false;
    float r[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) r[i][j] = s[i][j];
    for (int j = 0; j < 3; ++j) {
        const float n = (float)std::sqrt((double)r[0][j] * r[0][j] + (double)r[1][j] * r[1][j] + (double)r[2][j] * r[2][j]);
        if (n != 0.0f)
            for (int i = 0; i < 3; ++i) r[i][j] /= n;
    }
    float c[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) c[i][j] = r[i][0] * r[j][0] + r[i][1] * r[j][1] + r[i][2] * r[j][2];
    return is_identity<3>(c, 1.0e-4);
}

// sform_and_qform_are_very_similar (nifti.rs:1702-1722)
bool sform_qform_very_similar(const M44 s, const M44 q) {
    double sa[3][3], qa[3][3], su[3][3], sw[3], sv[3][3], qu[3][3], qw[3], qv[3][3];
    top33(s, sa);
    top33(q, qa);
    jacobi_svd<3>(sa, su, sw, sv);
    jacobi_svd<3>(qa, qu, qw, qv);
    float c[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) c[i][j] = (float)(su[i][0] * qu[j][0] + su[i][1] * qu[j][1] + su[i][2] * qu[j][2]);
    for (int i = 0; i < 3; ++i)
        if (std::fabs(sw[i] - qw[i]) > 1.0e-4) return false;
    if (!is_identity<3>(c, 1.0e-4)) return false;
    for (int i = 0; i < 3; ++i)
        if ((double)std::fabs(s[i][3] - q[i][3]) > 1.0e-4) return false;
    for (int j = 0; j < 4; ++j)
        if ((double)std::fabs(s[3][j] - q[3][j]) > 1.0e-4) return false;
    return true;
}

// ITK_NIFTI_SFORM_PERMISSIVE: on unless unset or NO / OFF / FALSE (nifti.rs:1611-1619)
bool sform_permissive() {
    const char* v = std::getenv("ITK_NIFTI_SFORM_PERMISSIVE");
    if (!v) return false;
    const std::string u = upper(v);
    return u != "NO" && u != "OFF" && u != "FALSE";
}

// the_mat (nifti.rs:1724-1768)
bool the_mat(const M44 s, const M44 q, int16_t scode, int16_t qcode, M44 out, std::string& why) {
    bool prefer_s = qform_sform_similar(s, q);
    if (!prefer_s || scode != XFORM_UNKNOWN) {
        if (sform_without_skew(s)) {
            const bool qk = qcode != XFORM_UNKNOWN, sk = scode != XFORM_UNKNOWN;
            if ((!qk && sk) || scode == XFORM_SCANNER_ANAT)
                prefer_s = true;
            else if (qk && sk)
                prefer_s = sform_qform_very_similar(s, q);
        } else if (sform_permissive()) {
            double a[3][3], u[3][3], w[3], v[3][3];
            top33(s, a);
            jacobi_svd<3>(a, u, w, v);
            if (w[2] > 1e-8) {
                std::memset(out, 0, sizeof(M44));
                for (int i = 0; i < 3; ++i)
                    for (int j = 0; j < 3; ++j) out[i][j] = (float)(u[i][0] * v[j][0] + u[i][1] * v[j][1] + u[i][2] * v[j][2]);
                for (int i = 0; i < 3; ++i) out[i][3] = s[i][3];
                for (int j = 0; j < 4; ++j) out[3][j] = s[3][j];
                return true;
            }
        }
    }
    if (prefer_s) {
        std::memcpy(out, s, sizeof(M44));
        return true;
    }
    if (qcode != XFORM_UNKNOWN) {
        std::memcpy(out, q, sizeof(M44));
        return true;
    }
    why = "no orthonormal definition of the direction cosines (neither the sform nor the qform)";
    return false;
}

// ---- the image ----

struct Nifti {
    mi_geometry geo{};
    int16_t datatype = 0;
    int nbyper = 0;
    bool swap = false;
    bool rescale = false;
    double slope = 1.0, inter = 0.0;
    int64_t nvox = 0;
    std::string img;       // the file holding the voxels
    int64_t offset = 0;    // where they start (negative: at the end of the file)
};

mi_dtype dtype_of(int16_t dt) {
    switch (dt) {
        case DT_UINT8: return MI_U8;
        case DT_INT8: return MI_I8;
        case DT_UINT16: return MI_U16;
        case DT_INT16: return MI_I16;
        case DT_UINT32: return MI_U32;
        case DT_INT32: return MI_I32;
        case DT_UINT64: return MI_U64;
        case DT_INT64: return MI_I64;
        case DT_FLOAT32: return MI_F32;
        default: return MI_F64;
    }
}

int bytes_of(int16_t dt) {
    switch (dt) {
        case DT_UINT8: case DT_INT8: return 1;
        case DT_UINT16: case DT_INT16: return 2;
        case DT_UINT32: case DT_INT32: case DT_FLOAT32: return 4;
        case DT_UINT64: case DT_INT64: case DT_FLOAT64: return 8;
        default: return 0;
    }
}

bool read_info(const std::string& path, Nifti& n, Fail& fail) {
    std::string hdr;
    if (!find_hdr_name(path, hdr)) {
        fail = {MI_ERR_INVALID_ARGUMENT, path + " is not recognised as a NIfTI file"};
        return false;
    }
    std::string bytes;
    if (!read_bytes(hdr, bytes, HDR)) {
        fail = {MI_ERR_INVALID_ARGUMENT, "cannot read " + hdr};
        return false;
    }
    Header h;
    std::string why;
    if (!parse_header(bytes, h, n.swap, why)) {
        fail = {MI_ERR_INVALID_ARGUMENT, "NIfTI header: " + why};
        return false;
    }
    // nifti_convert_nhdr2nim (nifti.rs:1090-1310)
    if (h.datatype == 0 || h.datatype == 1) {
        fail = {MI_ERR_INVALID_ARGUMENT, "NIfTI header: bad datatype"};
        return false;
    }
    if (h.dim[1] <= 0) {
        fail = {MI_ERR_INVALID_ARGUMENT, "NIfTI header: bad dim[1]"};
        return false;
    }
    const bool is_nifti = nifti_version(h.magic) != 0;
    const int dim0 = h.dim[0];
    for (int i = 2; i <= std::min(dim0, 7); ++i)
        if (h.dim[i] <= 0) h.dim[i] = 1;
    for (int i = dim0 + 1; i <= 7; ++i)
        if (h.dim[i] != 1 && h.dim[i] != 0) h.dim[i] = 1;
    for (int i = 1; i <= std::min(dim0, 7); ++i)
        if (h.pixdim[i] == 0.0f || !std::isfinite(h.pixdim[i])) h.pixdim[i] = 1.0f;
    const bool onefile = is_nifti && h.magic[1] == '+';
    int ftype = is_nifti ? (onefile ? FTYPE_NIFTI1_1 : FTYPE_NIFTI1_2) : FTYPE_ANALYZE;
    n.nvox = 1;
    for (int i = 1; i <= std::min(dim0, 7); ++i) n.nvox *= (int64_t)h.dim[i];
    M44 q, s;
    int16_t qcode = XFORM_UNKNOWN, scode = XFORM_UNKNOWN;
    if (!is_nifti || h.qform_code <= 0) {
        std::memset(q, 0, sizeof(M44));
        q[0][0] = h.pixdim[1];
        q[1][1] = h.pixdim[2];
        q[2][2] = h.pixdim[3];
        q[3][3] = 1.0f;
    } else {
        quatern_to_mat44(fixed_f32(h.qb), fixed_f32(h.qc), fixed_f32(h.qd), fixed_f32(h.qx), fixed_f32(h.qy),
                         fixed_f32(h.qz), h.pixdim[1], h.pixdim[2], h.pixdim[3], h.pixdim[0] < 0.0f ? -1.0f : 1.0f, q);
        qcode = h.qform_code;
    }
    std::memset(s, 0, sizeof(M44));
    if (is_nifti && h.sform_code > 0) {
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 4; ++c) s[r][c] = h.srow[r][c];
        s[3][3] = 1.0f;
        scode = h.sform_code;
    }
    const int iname_offset = onefile ? std::max((int)h.vox_offset, HDR) : (int)h.vox_offset;
    const std::string iname = make_img_name(hdr, is_gz(hdr));
    if (iname == hdr)
        ftype = FTYPE_NIFTI1_1;
    else if (ftype == FTYPE_NIFTI1_1)
        ftype = FTYPE_NIFTI1_2;
    const int16_t intent = is_nifti ? h.intent_code : 0;
    // dimension and pixel kind (nifti.rs read_info, :2020-2080)
    if (intent == INTENT_GENMATRIX || intent == INTENT_SYMMATRIX || intent == INTENT_DISPVECT ||
        intent == INTENT_VECTOR) {
        fail = {MI_ERR_INVALID_ARGUMENT, "vector and matrix NIfTI images (intent " + std::to_string(intent) +
                                             ") are not read: the metric takes scalar volumes"};
        return false;
    }
    int realdim = dim0;
    while (realdim > 3 && h.dim[realdim] == 1) --realdim;
    if (realdim != 3) {
        fail = {MI_ERR_INVALID_ARGUMENT, "a " + std::to_string(realdim) + "-D NIfTI image: only 3-D volumes are read"};
        return false;
    }
    if (h.datatype == DT_COMPLEX64 || h.datatype == DT_COMPLEX128 || h.datatype == DT_RGB24 ||
        h.datatype == DT_RGBA32) {
        fail = {MI_ERR_UNSUPPORTED_PIXEL_TYPE, "complex and RGB NIfTI datatypes are not scalar"};
        return false;
    }
    n.datatype = h.datatype;
    n.nbyper = bytes_of(h.datatype);
    if (n.nbyper == 0) {
        fail = {MI_ERR_INVALID_ARGUMENT, "unsupported NIfTI datatype " + std::to_string(h.datatype)};
        return false;
    }
    // rescale (nifti.rs:2085-2099)
    if (ftype == FTYPE_ANALYZE || !is_nifti) {
        n.slope = 1.0;
        n.inter = 0.0;
    } else {
        n.slope = (double)fixed_f32(h.scl_slope);
        if (std::fabs(n.slope) < DBL_EPSILON) n.slope = 1.0;
        n.inter = (double)fixed_f32(h.scl_inter);
    }
    n.rescale = std::fabs(n.slope) > DBL_EPSILON &&
                (std::fabs(n.slope - 1.0) > DBL_EPSILON || std::fabs(n.inter) > DBL_EPSILON);
    const int xyz_units = is_nifti ? (h.xyzt_units & 0x07) : 0;
    const double sscale = xyz_units == 1 ? 1e3 : (xyz_units == 3 ? 1e-3 : 1.0);
    for (int d = 0; d < 3; ++d) {
        n.geo.size[d] = h.dim[d + 1];
        n.geo.spacing[d] = (double)h.pixdim[d + 1] * sscale;
        n.geo.origin[d] = 0.0;
    }
    for (int i = 0; i < 9; ++i) n.geo.direction[i] = i % 4 == 0 ? 1.0 : 0.0;
    if (qcode != XFORM_UNKNOWN || scode != XFORM_UNKNOWN) {
        // SetImageIOOrientationFromNIfTI (nifti.rs:1795-1876): RAS+ → LPS
        M44 m;
        if (!the_mat(s, q, scode, qcode, m, why)) {
            fail = {MI_ERR_INVALID_ARGUMENT, "NIfTI header: " + why};
            return false;
        }
        n.geo.origin[0] = -(double)m[0][3] * sscale;
        n.geo.origin[1] = -(double)m[1][3] * sscale;
        n.geo.origin[2] = (double)m[2][3] * sscale;
        for (int d = 0; d < 3; ++d) {
            double ax[3] = {-(double)m[0][d], -(double)m[1][d], (double)m[2][d]};
            const double sum = ax[0] * ax[0] + ax[1] * ax[1] + ax[2] * ax[2];
            if (sum != 0.0) {
                const double r = std::sqrt(sum);
                for (double& x : ax) x /= r;
            }
            for (int j = 0; j < 3; ++j) n.geo.direction[j * 3 + d] = ax[j];
        }
    }
    if (!find_img_name(iname, ftype, n.img)) {
        fail = {MI_ERR_INVALID_ARGUMENT, "the voxel file of " + hdr + " is missing (" + iname + ")"};
        return false;
    }
    n.offset = iname_offset;
    return true;
}

template <class T>
void decode(const char* src, int64_t n, bool swap, float* dst, bool rescale, double slope, double inter) {
    for (int64_t i = 0; i < n; ++i) {
        unsigned char b[sizeof(T)];
        std::memcpy(b, src + i * (int64_t)sizeof(T), sizeof(T));
        if (swap)
            for (size_t a = 0, z = sizeof(T) - 1; a < z; ++a, --z) std::swap(b[a], b[z]);
        T x;
        std::memcpy(&x, b, sizeof(T));
        if (!rescale)
            dst[i] = (float)(double)x;  // the upload cast of every scalar type
        else if (std::is_same<T, double>::value)
            dst[i] = (float)((double)x * slope + inter);  // f64 data: rescaled in f64
        else
            // integers are cast to f32 first; f32 data rescaled through f64, stored as f32
            dst[i] = (float)((double)(float)x * slope + inter);
    }
}

bool read_voxels(const Nifti& n, float* dst, Fail& fail) {
    std::string raw;
    if (!read_bytes(n.img, raw)) {
        fail = {MI_ERR_INVALID_ARGUMENT, "cannot read " + n.img};
        return false;
    }
    const int64_t ntot = n.nvox * n.nbyper;
    const int64_t off = n.offset < 0 ? std::max<int64_t>((int64_t)raw.size() - ntot, 0) : n.offset;
    if ((int64_t)raw.size() < off + ntot) {
        fail = {MI_ERR_INVALID_ARGUMENT, "NIfTI voxel data is truncated"};
        return false;
    }
    const char* p = raw.data() + off;
    const int64_t nv = n.geo.size[0] * n.geo.size[1] * n.geo.size[2];
    switch (n.datatype) {
        case DT_UINT8: decode<uint8_t>(p, nv, n.swap, dst, n.rescale, n.slope, n.inter); break;
        case DT_INT8: decode<int8_t>(p, nv, n.swap, dst, n.rescale, n.slope, n.inter); break;
        case DT_UINT16: decode<uint16_t>(p, nv, n.swap, dst, n.rescale, n.slope, n.inter); break;
        case DT_INT16: decode<int16_t>(p, nv, n.swap, dst, n.rescale, n.slope, n.inter); break;
        case DT_UINT32: decode<uint32_t>(p, nv, n.swap, dst, n.rescale, n.slope, n.inter); break;
        case DT_INT32: decode<int32_t>(p, nv, n.swap, dst, n.rescale, n.slope, n.inter); break;
        case DT_UINT64: decode<uint64_t>(p, nv, n.swap, dst, n.rescale, n.slope, n.inter); break;
        case DT_INT64: decode<int64_t>(p, nv, n.swap, dst, n.rescale, n.slope, n.inter); break;
        case DT_FLOAT32: decode<float>(p, nv, n.swap, dst, n.rescale, n.slope, n.inter); break;
        default: decode<double>(p, nv, n.swap, dst, n.rescale, n.slope, n.inter); break;
    }
    return true;
}

}  // namespace
}  // namespace mi

extern "C" {

mi_status mi_image_read_nifti_host(const char* path, mi_geometry* geometry, float* dst, size_t n_elements) {
    if (!path || !geometry) return MI_ERR_INVALID_ARGUMENT;
    mi::Nifti n;
    mi::Fail fail{MI_OK, ""};
    if (!mi::read_info(path, n, fail)) return fail.s;
    *geometry = n.geo;
    if (!dst) return MI_OK;  // geometry only
    const size_t nv = (size_t)(n.geo.size[0] * n.geo.size[1] * n.geo.size[2]);
    if (n_elements < nv) return MI_ERR_INVALID_ARGUMENT;
    if (!mi::read_voxels(n, dst, fail)) return fail.s;
    return MI_OK;
}

mi_status mi_image_read_nifti(mi_context* ctx, const char* path, mi_image** out) {
    if (!ctx || !path || !out) return MI_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    mi::Nifti n;
    mi::Fail fail{MI_OK, ""};
    if (!mi::read_info(path, n, fail)) return mi::set_error(ctx, fail.s, fail.why);
    std::vector<float> v((size_t)(n.geo.size[0] * n.geo.size[1] * n.geo.size[2]));
    if (!mi::read_voxels(n, v.data(), fail)) return mi::set_error(ctx, fail.s, fail.why);
    return mi_image_upload(ctx, v.data(), MI_F32, &n.geo, out);
}

}  // extern "C"
