// OOMMF OVF 2.0 files of vector data (rectangular meshes, valuedim 3), host only.
//
// Reading follows OVF2::Read_OVF2_VEC (Boris/OVF2_Handlers.cpp:364):
//   - the first line must be "# OOMMF OVF 2.0" (else a version mismatch, BM_EUNSUPPORTED);
//   - header lines are recognised by the keys "# meshtype: ", "# meshunit: ", "# valuedim: ",
//     "# xmin: " .. "# zmax: ", "# xnodes: " .. "# znodes: ", "# xstepsize: " .. "# zstepsize: "
//     (constructor, :4); every other line is ignored; a trailing carriage return is dropped (:219);
//   - meshtype must be "rectangular", meshunit "m" or "nm" (lengths scale by 1 or 1e-9, applied to
//     the values that follow it), valuedim "3";
//   - "# Begin: data " (compared lower-case) followed by "binary 4", "binary 8" or "text" starts
//     the data; before it the mesh type, valuedim, rectangle, nodes and step sizes must all be set;
//   - binary data starts with the check value 1234567.0 (float) or 123456789012345.0 (double);
//   - the node counts must equal the ones the rectangle and step sizes give (VEC::resize(h, rect),
//     n = max(1, round(size / h)), BorisLib/VEC_mng.h:39,154);
//   - values follow x fastest, then y, then z; text rows hold at least three space- or
//     tab-separated numbers (a shorter row leaves that cell at zero, :666).
// Unlike the reference, a file that ends before all values are read is refused (BM_EINVAL) rather
// than leaving the remaining cells unset.
//
// Writing follows OVF2::Write_OVF2_VEC (Boris/OVF2_Handlers.cpp:701): the same header lines, in the
// same order, numbers printed with 6 significant digits (the reference's ToString precision,
// BorisLib/Types_Conversion.h:110), "# Title: " followed by the file name without its directory,
// values divided by `norm`, data types "bin4", "bin8" and "text".
//
// Mapping to other dimensions follows VEC::mapmesh_newdims (BorisLib/VEC_mng.h:9): destination
// cell (i, j, k) takes source cell (floor(i * nsx / ndx), floor(j * nsy / ndy), floor(k * nsz / ndz)).
// Renormalisation follows VEC::renormalize (BorisLib/VEC_oper.h:45): every vector longer than
// 1e-12 is scaled to the given length.
#include "boris_b200.h"

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

int bm_set_error(int code, const std::string &msg);

namespace {

const char *K_VERSION = "# OOMMF OVF 2.0";
const char *K_BEGIN_DATA = "# Begin: data ";
const char *K_END_DATA = "# End: data ";

std::string lower(std::string s)
{
    for (auto &ch : s) ch = (char)std::tolower((unsigned char)ch);
    return s;
}

// value after `key` when the line contains it (the key is taken to start the line, as in the
// reference, which cuts the key's length off the front)
bool keyed(const std::string &line, const char *key, std::string &value)
{
    if (line.find(key) == std::string::npos) return false;
    size_t L = std::strlen(key);
    value = line.size() > L ? line.substr(L) : std::string();
    return true;
}

bool read_line(std::istream &in, std::string &line)
{
    if (!std::getline(in, line)) return false;
    if (!line.empty() && line.back() == '\r') line.pop_back();
    return true;
}

struct Header {
    bool rectangular = false;
    double unit = 1.0;
    int valuedim = 0;
    double s[3] = {0, 0, 0}, e[3] = {0, 0, 0}, h[3] = {0, 0, 0};
    int n[3] = {0, 0, 0};
    int bytes = 0;   // 4, 8, or 1 for text
};

// 0: bad line, 1: fine, 2: start of data
int scan(const std::string &line, Header &H)
{
    static const char *rect_keys[6] = {"# xmin: ", "# ymin: ", "# zmin: ", "# xmax: ", "# ymax: ", "# zmax: "};
    static const char *node_keys[3] = {"# xnodes: ", "# ynodes: ", "# znodes: "};
    static const char *step_keys[3] = {"# xstepsize: ", "# ystepsize: ", "# zstepsize: "};
    std::string v;
    if (keyed(line, "# meshtype: ", v)) {
        if (v != "rectangular") return 0;
        H.rectangular = true;
        return 1;
    }
    if (keyed(line, "# meshunit: ", v)) {
        if (v == "m") H.unit = 1.0;
        else if (v == "nm") H.unit = 1e-9;
        else return 0;
        return 1;
    }
    if (keyed(line, "# valuedim: ", v)) {
        if (v != "3") return 0;
        H.valuedim = 3;
        return 1;
    }
    for (int a = 0; a < 6; a++)
        if (keyed(line, rect_keys[a], v)) {
            (a < 3 ? H.s[a] : H.e[a - 3]) = std::strtod(v.c_str(), nullptr) * H.unit;
            return 1;
        }
    for (int a = 0; a < 3; a++)
        if (keyed(line, node_keys[a], v)) {
            H.n[a] = (int)std::strtol(v.c_str(), nullptr, 10);
            return 1;
        }
    for (int a = 0; a < 3; a++)
        if (keyed(line, step_keys[a], v)) {
            H.h[a] = std::strtod(v.c_str(), nullptr) * H.unit;
            return 1;
        }
    std::string low = lower(line);
    if (low.find(lower(K_BEGIN_DATA)) != std::string::npos) {
        std::string t = low.size() > std::strlen(K_BEGIN_DATA) ? low.substr(std::strlen(K_BEGIN_DATA)) : std::string();
        if (t == "binary 4") H.bytes = 4;
        else if (t == "binary 8") H.bytes = 8;
        else if (t == "text") H.bytes = 1;
        else return 1;   // an unknown data kind is not a data start, as in the reference
        return 2;
    }
    return 1;
}

bool header_complete(const Header &H)
{
    // the reference's vector equality has a 1e-12 tolerance (BorisLib/Types_VAL.h:500)
    bool rect_null = true, n_zero = true, h_zero = true;
    for (int a = 0; a < 3; a++) {
        if (std::fabs(H.s[a]) >= 1e-12 || std::fabs(H.e[a]) >= 1e-12) rect_null = false;
        if (H.n[a] != 0) n_zero = false;
        if (std::fabs(H.h[a]) >= 1e-12) h_zero = false;
    }
    return H.rectangular && H.valuedim == 3 && !rect_null && !n_zero && !h_zero && H.bytes;
}

// node counts the rectangle and step sizes give: max(1, round(size / h))
bool nodes_match(const Header &H)
{
    for (int a = 0; a < 3; a++) {
        if (H.h[a] == 0.0 || H.n[a] < 1) return false;
        double q = std::round((H.e[a] - H.s[a]) / H.h[a]);
        long long na = q < 1 ? 1 : (long long)q;
        if (na != H.n[a]) return false;
    }
    return true;
}

std::string g6(double v)
{
    char b[64];
    std::snprintf(b, sizeof b, "%.6g", v);
    return b;
}

std::string base_name(const std::string &path)
{
    size_t p = path.find_last_of("/\\");
    return p == std::string::npos ? path : path.substr(p + 1);
}

}  // namespace

extern "C" int bm_ovf2_read(const char *path, int *n3, double *h3, double *rect6, double *data, long long capacity)
{
    if (!path) return bm_set_error(BM_EINVAL, "bm_ovf2_read: null path");
    std::ifstream in(path, std::ios::in | std::ios::binary);
    if (!in.is_open()) return bm_set_error(BM_EINVAL, std::string("bm_ovf2_read: could not open ") + path);
    std::string line;
    if (!read_line(in, line) || line != K_VERSION)
        return bm_set_error(BM_EUNSUPPORTED, "bm_ovf2_read: not an OOMMF OVF 2.0 file (first line)");
    Header H;
    int st = 1;
    while (read_line(in, line)) {
        st = scan(line, H);
        if (st == 0) return bm_set_error(BM_EINVAL, "bm_ovf2_read: unsupported or malformed header line: " + line);
        if (st == 2) break;
    }
    if (st != 2) return bm_set_error(BM_EINVAL, "bm_ovf2_read: no data segment");
    if (!header_complete(H)) return bm_set_error(BM_EINVAL, "bm_ovf2_read: incomplete header (meshtype, valuedim, rectangle, nodes, step sizes)");
    if (!nodes_match(H)) return bm_set_error(BM_EINVAL, "bm_ovf2_read: node counts do not match the rectangle and step sizes");
    if (H.bytes == 4) {
        float chk = 0;
        in.read(reinterpret_cast<char *>(&chk), 4);
        if (!in || chk != 1234567.0f) return bm_set_error(BM_EINVAL, "bm_ovf2_read: binary 4 check value missing");
    } else if (H.bytes == 8) {
        double chk = 0;
        in.read(reinterpret_cast<char *>(&chk), 8);
        if (!in || chk != 123456789012345.0) return bm_set_error(BM_EINVAL, "bm_ovf2_read: binary 8 check value missing");
    }
    if (n3) for (int a = 0; a < 3; a++) n3[a] = H.n[a];
    // the step sizes the reference keeps: size / n (VEC::set_n_adjust_h)
    if (h3) for (int a = 0; a < 3; a++) h3[a] = (H.e[a] - H.s[a]) / H.n[a];
    if (rect6) for (int a = 0; a < 3; a++) { rect6[a] = H.s[a]; rect6[3 + a] = H.e[a]; }
    if (!data) return 0;
    long long ncell = (long long)H.n[0] * H.n[1] * H.n[2];
    if (capacity < 3 * ncell) return bm_set_error(BM_EINVAL, "bm_ovf2_read: data buffer too small");
    if (H.bytes == 4) {
        std::vector<float> buf(3 * (size_t)ncell);
        in.read(reinterpret_cast<char *>(buf.data()), (std::streamsize)(buf.size() * 4));
        if (!in) return bm_set_error(BM_EINVAL, "bm_ovf2_read: file ends inside the data");
        for (size_t i = 0; i < buf.size(); i++) data[i] = buf[i];
    } else if (H.bytes == 8) {
        in.read(reinterpret_cast<char *>(data), (std::streamsize)(3 * ncell * 8));
        if (!in) return bm_set_error(BM_EINVAL, "bm_ovf2_read: file ends inside the data");
    } else {
        for (long long c = 0; c < ncell; c++) {
            if (!read_line(in, line)) return bm_set_error(BM_EINVAL, "bm_ovf2_read: file ends inside the data");
            double v[3];
            int got = 0;
            const char *p = line.c_str();
            while (got < 3) {
                while (*p == ' ' || *p == '\t') p++;
                if (!*p) break;
                char *q = nullptr;
                v[got] = std::strtod(p, &q);
                if (q == p) break;
                got++;
                p = q;
            }
            if (got == 3) { data[3 * c] = v[0]; data[3 * c + 1] = v[1]; data[3 * c + 2] = v[2]; }
            else { data[3 * c] = data[3 * c + 1] = data[3 * c + 2] = 0.0; }
        }
    }
    return 0;
}

extern "C" int bm_ovf2_write(const char *path, const int *n3, const double *h3, const double *origin3,
                             const double *data, const char *data_type, double norm)
{
    if (!path || !n3 || !h3 || !data) return bm_set_error(BM_EINVAL, "bm_ovf2_write: null argument");
    std::string kind = data_type ? data_type : "bin8";
    std::string tag;
    if (kind == "bin4") tag = "binary 4";
    else if (kind == "bin8") tag = "binary 8";
    else if (kind == "text") tag = "text";
    else return bm_set_error(BM_EINVAL, "bm_ovf2_write: data type must be bin4, bin8 or text");
    for (int a = 0; a < 3; a++)
        if (n3[a] < 1 || !(h3[a] > 0)) return bm_set_error(BM_EINVAL, "bm_ovf2_write: sizes and cellsizes must be positive");
    if (!(norm != 0.0) || !std::isfinite(norm)) return bm_set_error(BM_EINVAL, "bm_ovf2_write: norm must be finite and non-zero");
    std::ofstream out(path, std::ios::out | std::ios::binary | std::ios::trunc);
    if (!out.is_open()) return bm_set_error(BM_EINVAL, std::string("bm_ovf2_write: could not open ") + path);
    double s[3], e[3];
    for (int a = 0; a < 3; a++) {
        s[a] = origin3 ? origin3[a] : 0.0;
        e[a] = s[a] + n3[a] * h3[a];
    }
    std::string hd;
    hd += std::string(K_VERSION) + "\n#\n# Segment count: 1\n#\n# Begin: Segment\n# Begin: Header\n#\n";
    hd += "# Title: " + base_name(path) + "\n#\n";
    hd += "# meshunit: m\n#\n# meshtype: rectangular\n#\n";
    hd += "# xmin: " + g6(s[0]) + "\n# ymin: " + g6(s[1]) + "\n# zmin: " + g6(s[2]) + "\n";
    hd += "# xmax: " + g6(e[0]) + "\n# ymax: " + g6(e[1]) + "\n# zmax: " + g6(e[2]) + "\n#\n";
    hd += "# xnodes: " + std::to_string(n3[0]) + "\n# ynodes: " + std::to_string(n3[1]) + "\n# znodes: " +
          std::to_string(n3[2]) + "\n#\n";
    hd += "# xstepsize: " + g6(h3[0]) + "\n# ystepsize: " + g6(h3[1]) + "\n# zstepsize: " + g6(h3[2]) + "\n#\n";
    hd += "# valuedim: 3\n#\n# End: Header\n#\n";
    hd += std::string(K_BEGIN_DATA) + tag + "\n";
    out << hd;
    long long ncell = (long long)n3[0] * n3[1] * n3[2];
    if (kind == "bin4") {
        std::vector<float> buf(1 + 3 * (size_t)ncell);
        buf[0] = 1234567.0f;
        for (long long i = 0; i < 3 * ncell; i++) buf[1 + i] = (float)(data[i] / norm);
        out.write(reinterpret_cast<const char *>(buf.data()), (std::streamsize)(buf.size() * 4));
    } else if (kind == "bin8") {
        std::vector<double> buf(1 + 3 * (size_t)ncell);
        buf[0] = 123456789012345.0;
        for (long long i = 0; i < 3 * ncell; i++) buf[1 + i] = data[i] / norm;
        out.write(reinterpret_cast<const char *>(buf.data()), (std::streamsize)(buf.size() * 8));
    } else {
        std::string row;
        for (long long c = 0; c < ncell; c++) {
            row = g6(data[3 * c] / norm) + " " + g6(data[3 * c + 1] / norm) + " " + g6(data[3 * c + 2] / norm) + "\n";
            out << row;
        }
    }
    out << std::string(K_END_DATA) + tag + "\n# End: Segment\n";
    out.close();
    if (!out) return bm_set_error(BM_EINVAL, std::string("bm_ovf2_write: write failed for ") + path);
    return 0;
}

extern "C" int bm_map_cells(const double *src, const int *src_n3, double *dst, const int *dst_n3)
{
    if (!src || !dst || !src_n3 || !dst_n3) return bm_set_error(BM_EINVAL, "bm_map_cells: null argument");
    for (int a = 0; a < 3; a++)
        if (src_n3[a] < 1 || dst_n3[a] < 1) return bm_set_error(BM_EINVAL, "bm_map_cells: sizes must be >= 1");
    double r[3];
    for (int a = 0; a < 3; a++) r[a] = (double)src_n3[a] / dst_n3[a];
    for (int k = 0; k < dst_n3[2]; k++) {
        int sk = (int)std::floor(k * r[2]);
        for (int j = 0; j < dst_n3[1]; j++) {
            int sj = (int)std::floor(j * r[1]);
            for (int i = 0; i < dst_n3[0]; i++) {
                int si = (int)std::floor(i * r[0]);
                long long d = i + (long long)dst_n3[0] * (j + (long long)dst_n3[1] * k);
                long long s = si + (long long)src_n3[0] * (sj + (long long)src_n3[1] * sk);
                dst[3 * d] = src[3 * s];
                dst[3 * d + 1] = src[3 * s + 1];
                dst[3 * d + 2] = src[3 * s + 2];
            }
        }
    }
    return 0;
}

extern "C" int bm_renormalize(double *data, long long ncell, double length)
{
    if (!data || ncell < 0) return bm_set_error(BM_EINVAL, "bm_renormalize: bad argument");
    for (long long c = 0; c < ncell; c++) {
        double *v = data + 3 * c;
        double l = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        if (l > 1e-12) {   // IsNZ (BorisLib/Funcs_Aux_base.h:35)
            double f = length / l;
            v[0] *= f; v[1] *= f; v[2] *= f;
        }
    }
    return 0;
}
