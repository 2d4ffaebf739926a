// sdf.cpp -- snapshot and checkpoint files in the SDF ("self-describing
// file") format the reference writes its bodies in (nln/output.c:199-217
// writes the outbody records of nln/physics.h:49-58 with the descriptor
// OUTBODYDESC, nln/physics.h:62-110, through the 2hot SDF library, which
// is not vendored).  A file is an ASCII header of C-like declarations --
//     # SDF 1.0
//     parameter byteorder = 0x78563412;
//     int iter = 3;
//     double tpos = 0.25;
//     ...
//     struct {
//         float mass;
//         float x, y, z;
//         ...
//         int64_t ident;
//     }[1024];
//     #\f
//     # SDF-EOH
// -- followed by the packed little-endian records.  This writes and reads
// that layout: the records are outbody (mass, x y z, vx vy vz, with
// SAVE_ACC also ax ay az phi, int64 ident), the header scalars int,
// int64_t, float and double.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "nlnhost.h"

namespace {

thread_local std::string g_sdf_err;

int fail(const std::string &msg) {
    g_sdf_err = msg;
    return -1;
}

const char *type_name(int t) {
    switch (t) {
    case NLN_SDF_INT: return "int";
    case NLN_SDF_INT64: return "int64_t";
    case NLN_SDF_FLOAT: return "float";
    case NLN_SDF_DOUBLE: return "double";
    default: return nullptr;
    }
}

#pragma pack(push, 1)
struct OutBody {       // outbody without SAVE_ACC (nln/physics.h:49-58)
    float mass, pos[3], vel[3];
    int64_t ident;
};
struct OutBodyAcc {    // outbody with SAVE_ACC
    float mass, pos[3], vel[3], acc[3], phi;
    int64_t ident;
};
#pragma pack(pop)
static_assert(sizeof(OutBody) == 36 && sizeof(OutBodyAcc) == 52, "packed outbody");

const char *kBodyDesc =
    "struct {\n"
    "    float mass;\t\t\t/* mass of body */\n"
    "    float x, y, z;\t\t/* position of body */\n"
    "    float vx, vy, vz;\t\t/* velocity of body */\n"
    "    int64_t ident;\t\t/* unique? identifier */\n"
    "}";
const char *kBodyAccDesc =
    "struct {\n"
    "    float mass;\t\t\t/* mass of body */\n"
    "    float x, y, z;\t\t/* position of body */\n"
    "    float vx, vy, vz;\t\t/* velocity of body */\n"
    "    float ax, ay, az;\t\t/* acceleration */\n"
    "    float phi;\t\t\t/* potential */\n"
    "    int64_t ident;\t\t/* unique? identifier */\n"
    "}";

// the header's end: a form feed line, then the end-of-header mark
const char *kEOH = "#\f\n# SDF-EOH\n";

}  // namespace

struct nln_sdf {
    std::vector<std::string> keys;
    std::vector<int> types;
    std::vector<double> values;
    std::vector<std::string> fields;  // record fields in order
    int64_t nrec = 0;
    int save_acc = 0;
    std::vector<unsigned char> data;  // nrec packed records
};

extern "C" const char *nln_sdf_error(void) { return g_sdf_err.c_str(); }

extern "C" int nln_sdf_write(const char *path, int64_t n, const float *mass, const float *pos,
                             const float *vel, const float *acc_phi, const int64_t *ident,
                             int nkeys, const char *const *keys, const int *types,
                             const double *values) {
    if (!path || n < 0 || (n > 0 && (!mass || !pos || !vel || !ident)) || nkeys < 0)
        return fail("nln_sdf_write: bad arguments");
    FILE *f = std::fopen(path, "wb");
    if (!f)
        return fail(std::string("nln_sdf_write: cannot open ") + path);
    std::fprintf(f, "# SDF 1.0\nparameter byteorder = 0x78563412;\n");
    for (int k = 0; k < nkeys; k++) {
        const char *tn = type_name(types[k]);
        if (!tn || !keys[k] || !keys[k][0]) {
            std::fclose(f);
            return fail("nln_sdf_write: bad header entry");
        }
        if (types[k] == NLN_SDF_INT || types[k] == NLN_SDF_INT64)
            std::fprintf(f, "%s %s = %lld;\n", tn, keys[k], (long long)values[k]);
        else
            std::fprintf(f, "%s %s = %.17g;\n", tn, keys[k], values[k]);
    }
    std::fprintf(f, "%s[%lld];\n%s", acc_phi ? kBodyAccDesc : kBodyDesc, (long long)n, kEOH);
    const size_t rec = acc_phi ? sizeof(OutBodyAcc) : sizeof(OutBody);
    std::vector<unsigned char> buf(rec * 65536);
    for (int64_t b0 = 0; b0 < n; b0 += 65536) {
        const int64_t b1 = std::min<int64_t>(n, b0 + 65536);
        for (int64_t i = b0; i < b1; i++) {
            unsigned char *o = buf.data() + (i - b0) * rec;
            if (acc_phi) {
                OutBodyAcc r;
                r.mass = mass[i];
                for (int d = 0; d < 3; d++) {
                    r.pos[d] = pos[3 * i + d];
                    r.vel[d] = vel[3 * i + d];
                    r.acc[d] = acc_phi[4 * i + d];
                }
                r.phi = acc_phi[4 * i + 3];
                r.ident = ident[i];
                std::memcpy(o, &r, rec);
            } else {
                OutBody r;
                r.mass = mass[i];
                for (int d = 0; d < 3; d++) {
                    r.pos[d] = pos[3 * i + d];
                    r.vel[d] = vel[3 * i + d];
                }
                r.ident = ident[i];
                std::memcpy(o, &r, rec);
            }
        }
        if (std::fwrite(buf.data(), rec, (size_t)(b1 - b0), f) != (size_t)(b1 - b0)) {
            std::fclose(f);
            return fail("nln_sdf_write: short write");
        }
    }
    if (std::fclose(f) != 0)
        return fail("nln_sdf_write: close failed");
    return 0;
}

namespace {

// Header statements are ';'-terminated; comments /* */ are skipped.
std::string strip_comments(const std::string &h) {
    std::string o;
    for (size_t i = 0; i < h.size(); i++) {
        if (h.compare(i, 2, "/*") == 0) {
            const size_t e = h.find("*/", i + 2);
            if (e == std::string::npos)
                break;
            i = e + 1;
            continue;
        }
        o += h[i];
    }
    return o;
}

std::string trim(const std::string &s) {
    const size_t a = s.find_first_not_of(" \t\r\n");
    if (a == std::string::npos)
        return "";
    const size_t b = s.find_last_not_of(" \t\r\n");
    return s.substr(a, b - a + 1);
}

}  // namespace

extern "C" nln_sdf *nln_sdf_read(const char *path) {
    FILE *f = path ? std::fopen(path, "rb") : nullptr;
    if (!f) {
        fail(std::string("nln_sdf_read: cannot open ") + (path ? path : "(null)"));
        return nullptr;
    }
    std::string header;
    char line[4096];
    bool eoh = false;
    while (std::fgets(line, sizeof(line), f)) {
        if (std::strncmp(line, "# SDF-EOH", 9) == 0) {
            eoh = true;
            break;
        }
        if (line[0] == '#')
            continue;  // "# SDF 1.0", the form-feed line, comments
        header += line;
    }
    if (!eoh) {
        std::fclose(f);
        fail("nln_sdf_read: no end-of-header mark");
        return nullptr;
    }
    auto *s = new nln_sdf();
    const std::string h = strip_comments(header);
    auto bad = [&](const std::string &msg) -> nln_sdf * {
        delete s;
        std::fclose(f);
        fail(msg);
        return nullptr;
    };
    // scalar declarations "<type> <name> = <value>;" up to the record struct
    const size_t sp0 = h.find("struct");
    const std::string scalars = h.substr(0, sp0);
    size_t i = 0;
    while (i < scalars.size()) {
        const size_t semi = scalars.find(';', i);
        if (semi == std::string::npos)
            break;
        const std::string st = trim(scalars.substr(i, semi - i));
        i = semi + 1;
        const size_t eq = st.find('=');
        const size_t sp = st.find_first_of(" \t");
        if (st.empty() || eq == std::string::npos || sp == std::string::npos || sp > eq)
            continue;
        const std::string type = st.substr(0, sp);
        if (type == "parameter")
            continue;  // byteorder: this reader takes little-endian files
        const int t = type == "int" ? NLN_SDF_INT
                      : type == "int64_t" ? NLN_SDF_INT64
                      : type == "float" ? NLN_SDF_FLOAT
                      : type == "double" ? NLN_SDF_DOUBLE : -1;
        if (t < 0)
            continue;
        s->keys.push_back(trim(st.substr(sp + 1, eq - sp - 1)));
        s->types.push_back(t);
        s->values.push_back(std::strtod(trim(st.substr(eq + 1)).c_str(), nullptr));
    }
    // the record struct: "struct { <type> <name>, <name>; ... }[<n>];"
    if (sp0 == std::string::npos)
        return bad("nln_sdf_read: no record struct");
    const size_t open = h.find('{', sp0), close = h.find('}', sp0);
    const size_t lb = close == std::string::npos ? close : h.find('[', close);
    if (open == std::string::npos || close == std::string::npos || lb == std::string::npos ||
        open > close)
        return bad("nln_sdf_read: malformed record struct");
    s->nrec = std::strtoll(h.c_str() + lb + 1, nullptr, 10);
    const std::string members = h.substr(open + 1, close - open - 1);
    size_t m = 0;
    while (m < members.size()) {
        const size_t ms = members.find(';', m);
        if (ms == std::string::npos)
            break;
        const std::string decl = trim(members.substr(m, ms - m));
        m = ms + 1;
        if (decl.empty())
            continue;
        const size_t sp = decl.find_first_of(" \t");
        const std::string type = decl.substr(0, sp);
        if (type != "float" && type != "int64_t")
            return bad("nln_sdf_read: unsupported field type " + type);
        const std::string names = decl.substr(sp + 1);
        size_t c = 0;
        for (;;) {
            const size_t comma = names.find(',', c);
            const std::string nm =
                trim(names.substr(c, comma == std::string::npos ? std::string::npos : comma - c));
            if (!nm.empty())
                s->fields.push_back(nm);
            if (comma == std::string::npos)
                break;
            c = comma + 1;
        }
    }
    const std::vector<std::string> plain = {"mass", "x", "y", "z", "vx", "vy", "vz", "ident"};
    const std::vector<std::string> acc = {"mass", "x", "y", "z", "vx", "vy", "vz",
                                          "ax", "ay", "az", "phi", "ident"};
    if (s->fields != plain && s->fields != acc)
        return bad("nln_sdf_read: the records are not the outbody layout");
    if (s->nrec < 0)
        return bad("nln_sdf_read: bad record count");
    s->save_acc = s->fields == acc;
    const size_t rec = s->save_acc ? sizeof(OutBodyAcc) : sizeof(OutBody);
    s->data.resize(rec * (size_t)s->nrec);
    if (s->nrec > 0 && std::fread(s->data.data(), rec, (size_t)s->nrec, f) != (size_t)s->nrec)
        return bad("nln_sdf_read: the file ends before its records");
    std::fclose(f);
    return s;
}

extern "C" int64_t nln_sdf_count(const nln_sdf *s) { return s ? s->nrec : -1; }
extern "C" int nln_sdf_has_acc(const nln_sdf *s) { return s ? s->save_acc : 0; }
extern "C" int nln_sdf_nkeys(const nln_sdf *s) { return s ? (int)s->keys.size() : 0; }

extern "C" const char *nln_sdf_key(const nln_sdf *s, int k, int *type, double *value) {
    if (!s || k < 0 || k >= (int)s->keys.size())
        return nullptr;
    if (type)
        *type = s->types[k];
    if (value)
        *value = s->values[k];
    return s->keys[k].c_str();
}

extern "C" int nln_sdf_bodies(const nln_sdf *s, float *mass, float *pos, float *vel,
                              float *acc_phi, int64_t *ident) {
    if (!s)
        return fail("nln_sdf_bodies: no file");
    const size_t rec = s->save_acc ? sizeof(OutBodyAcc) : sizeof(OutBody);
    for (int64_t i = 0; i < s->nrec; i++) {
        const unsigned char *p = s->data.data() + rec * (size_t)i;
        if (s->save_acc) {
            OutBodyAcc r;
            std::memcpy(&r, p, rec);
            if (mass) mass[i] = r.mass;
            for (int d = 0; d < 3; d++) {
                if (pos) pos[3 * i + d] = r.pos[d];
                if (vel) vel[3 * i + d] = r.vel[d];
                if (acc_phi) acc_phi[4 * i + d] = r.acc[d];
            }
            if (acc_phi) acc_phi[4 * i + 3] = r.phi;
            if (ident) ident[i] = r.ident;
        } else {
            OutBody r;
            std::memcpy(&r, p, rec);
            if (mass) mass[i] = r.mass;
            for (int d = 0; d < 3; d++) {
                if (pos) pos[3 * i + d] = r.pos[d];
                if (vel) vel[3 * i + d] = r.vel[d];
            }
            if (ident) ident[i] = r.ident;
        }
    }
    return 0;
}

extern "C" void nln_sdf_free(nln_sdf *s) { delete s; }
