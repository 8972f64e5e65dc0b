// lp_io.cpp -- config XML, OBJ mesh and emitter-file readers without VTK.
//
// ReadConfig follows ReadXML::ExtractConfigVars and its helpers (src/IO/ReadXML.cpp:
// 93-168, 598-870, 965-1010): the same element names, atof/atoi conversions and
// defaults.  ReadObj follows vtkOBJReader as used by ImportExport::ImportObjModel
// (src/IO/ImportExport.cpp:341-392) and the region-id pass GenMediumIDsFromObjModel
// (src/IO/ImportExport.cpp:952-1053), whose boost::regex_match patterns are restated
// as small whole-line matchers.
#include <cctype>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <stdexcept>

#include "../../../include/lightprop.hpp"

namespace lp {
namespace {

// ---- a small XML element tree (elements, character data; no attributes needed)
struct XNode {
    std::string name, text;
    std::vector<XNode> kids;
    const XNode *child(const char *n) const
    {
        for (const auto &k : kids)
            if (k.name == n) return &k;
        return nullptr;
    }
};

struct XParser {
    const std::string &s;
    size_t i = 0;
    explicit XParser(const std::string &src) : s(src) {}
    [[noreturn]] void bad(const char *what)
    {
        throw std::runtime_error(std::string("config XML: ") + what + " at offset " + std::to_string(i));
    }
    void skip_misc()
    {
        for (;;) {
            while (i < s.size() && std::isspace((unsigned char)s[i])) ++i;
            if (s.compare(i, 4, "<!--") == 0) {
                size_t e = s.find("-->", i + 4);
                if (e == std::string::npos) bad("unterminated comment");
                i = e + 3;
            } else if (s.compare(i, 2, "<?") == 0) {
                size_t e = s.find("?>", i + 2);
                if (e == std::string::npos) bad("unterminated declaration");
                i = e + 2;
            } else if (s.compare(i, 2, "<!") == 0) {
                size_t e = s.find('>', i + 2);
                if (e == std::string::npos) bad("unterminated declaration");
                i = e + 1;
            } else {
                return;
            }
        }
    }
    XNode element()
    {
        if (i >= s.size() || s[i] != '<') bad("expected '<'");
        ++i;
        XNode n;
        while (i < s.size() && !std::isspace((unsigned char)s[i]) && s[i] != '>' && s[i] != '/') n.name += s[i++];
        size_t e = s.find('>', i);
        if (e == std::string::npos) bad("unterminated tag");
        bool empty = e > 0 && s[e - 1] == '/';
        i = e + 1;
        if (empty) return n;
        for (;;) {
            size_t lt = s.find('<', i);
            if (lt == std::string::npos) bad("missing closing tag");
            n.text += s.substr(i, lt - i);
            i = lt;
            if (s.compare(i, 4, "<!--") == 0) {
                skip_misc();
                continue;
            }
            if (s.compare(i, 2, "</") == 0) {
                size_t ce = s.find('>', i);
                if (ce == std::string::npos) bad("unterminated closing tag");
                i = ce + 1;
                break;
            }
            n.kids.push_back(element());
        }
        // trim character data
        size_t a = 0, b = n.text.size();
        while (a < b && std::isspace((unsigned char)n.text[a])) ++a;
        while (b > a && std::isspace((unsigned char)n.text[b - 1])) --b;
        n.text = n.text.substr(a, b - a);
        return n;
    }
};

// Whole-line matchers with the semantics of the reference's boost::regex_match patterns
// (ImportExport.cpp:965-968, 398): \w = [A-Za-z0-9_], \d = [0-9].
bool is_word(char c) { return std::isalnum((unsigned char)c) || c == '_'; }
bool all_of(const std::string &s, size_t a, size_t b, bool (*pred)(char))
{
    if (a >= b) return false;
    for (size_t i = a; i < b; ++i)
        if (!pred(s[i])) return false;
    return true;
}
bool is_digit(char c) { return c >= '0' && c <= '9'; }
// "^o (\w+)"
bool match_object(const std::string &l, std::string &name)
{
    if (l.size() < 3 || l[0] != 'o' || l[1] != ' ' || !all_of(l, 2, l.size(), is_word)) return false;
    name = l.substr(2);
    return true;
}
// "^f (.+)"
bool match_face(const std::string &l) { return l.size() >= 3 && l[0] == 'f' && l[1] == ' '; }
// "^g (\d+)$" (kind 1) and "^g (\d+)\_(\w+)" (kind 2)
int match_group(const std::string &l, int &outer, std::string &surf)
{
    if (l.size() < 3 || l[0] != 'g' || l[1] != ' ') return 0;
    size_t i = 2;
    while (i < l.size() && is_digit(l[i])) ++i;
    if (i == 2) return 0;
    outer = std::atoi(l.substr(2, i - 2).c_str());
    if (i == l.size()) return 1;
    if (l[i] != '_' || !all_of(l, i + 1, l.size(), is_word)) return 0;
    surf = l.substr(i + 1);
    return 2;
}
// "^(\d+\.?\d*) (\d+\.?\d*)$"
bool match_number(const std::string &s, size_t a, size_t b)
{
    size_t i = a;
    while (i < b && is_digit(s[i])) ++i;
    if (i == a) return false;
    if (i < b && s[i] == '.') ++i;
    while (i < b && is_digit(s[i])) ++i;
    return i == b;
}
bool match_emitter_line(const std::string &l, float &a, float &b)
{
    size_t sp = l.find(' ');
    if (sp == std::string::npos || !match_number(l, 0, sp) || !match_number(l, sp + 1, l.size())) return false;
    a = (float)std::atof(l.substr(0, sp).c_str());
    b = (float)std::atof(l.substr(sp + 1).c_str());
    return true;
}

float fval(const XNode *n, float d = 0.0f) { return n ? (float)std::atof(n->text.c_str()) : d; }
int ival(const XNode *n, int d = 0) { return n ? std::atoi(n->text.c_str()) : d; }

std::string dir_of(const std::string &p)
{
    size_t k = p.find_last_of('/');
    return k == std::string::npos ? std::string(".") : p.substr(0, k);
}
std::string base_of(const std::string &p)
{
    size_t k = p.find_last_of('/');
    return k == std::string::npos ? p : p.substr(k + 1);
}
bool exists(const std::string &p)
{
    std::ifstream f(p);
    return (bool)f;
}
// The shipped configs carry absolute paths of the author's machine; fall back to the
// file of the same name next to the config.
std::string resolve(const std::string &p, const std::string &cfgdir)
{
    if (p.empty() || exists(p)) return p;
    std::string q = cfgdir + "/" + base_of(p);
    return exists(q) ? q : p;
}

void read_tissue(const XNode &t, std::vector<Tissue> &out)
{
    // ReadXML::ExtractTissue (ReadXML.cpp:965-1010): fields keyed by <ID>
    Tissue x;
    x.id = ival(t.child("ID"));
    if (const XNode *n = t.child("name")) x.name = n->text;
    x.g = fval(t.child("anisotropy"));
    x.mua = fval(t.child("mua"));
    x.mus = fval(t.child("mus"));
    x.n = fval(t.child("refraction"), 1.0f);
    if (x.id < 0 || x.id > 1000) throw std::runtime_error("config: tissue ID out of range");
    if ((int)out.size() <= x.id) out.resize(x.id + 1);
    out[x.id] = x;
}

}  // namespace

Config ReadConfig(const std::string &path)
{
    std::ifstream f(path);
    if (!f) throw std::runtime_error("config: cannot open " + path);
    std::stringstream ss;
    ss << f.rdbuf();
    std::string src = ss.str();
    XParser p(src);
    p.skip_misc();
    XNode root = p.element();
    Config c;
    const std::string cfgdir = dir_of(path);
    for (const XNode &e : root.kids) {
        if (e.name == "modelfile") {
            c.modelfile = e.text;
        } else if (e.name == "model") {
            for (const XNode &m : e.kids) {
                if (m.name == "modelfile") c.modelfile = m.text;
                else if (m.name == "PixelPerUnit") c.ppu = fval(&m, 1.0f);
                else if (m.name == "dimensions") {
                    c.dims[0] = fval(m.child("x"), 1.0f);
                    c.dims[1] = fval(m.child("y"), 1.0f);
                    c.dims[2] = fval(m.child("z"), 1.0f);
                } else if (m.name == "tissueList") {
                    for (const XNode &t : m.kids)
                        if (t.name == "tissue") read_tissue(t, c.tissues);
                }
            }
        } else if (e.name == "Emittermodel") {
            for (const XNode &m : e.kids) {
                if (m.name == "file") c.emitterfile = m.text;
                else if (m.name == "position") {
                    // ReadXML.cpp:740-744 reads the first three nested elements in order
                    for (int k = 0; k < 3 && k < (int)m.kids.size(); ++k) c.emitter_pos[k] = fval(&m.kids[k]);
                } else if (m.name == "distance") c.emitter_distance = fval(&m);
                else if (m.name == "heading") {
                    for (int k = 0; k < 3 && k < (int)m.kids.size(); ++k) c.emitter_heading[k] = fval(&m.kids[k]);
                }
            }
        } else if (e.name == "SimulationParams") {
            for (const XNode &m : e.kids) {
                if (m.name == "numberOfPhotons") c.numberOfPhotons = std::atoll(m.text.c_str());
                else if (m.name == "numPhotonsInteractions") c.numPhotonsInteractions = ival(&m);
                else if (m.name == "chance") c.chance = fval(&m);
                else if (m.name == "weightThreshold") c.weightThreshold = fval(&m);
            }
        } else if (e.name == "saveLogFiles") {
            c.saveLogFiles = ival(&e) != 0;
        } else if (e.name == "saveDir") {
            c.saveDir = e.text;
        } else if (e.name == "analyse") {
            if (const XNode *b = e.child("boundaries"))
                for (const XNode &s : b->kids)
                    if (s.name == "surfName") c.surfNames.push_back(s.text);
        } else if (e.name == "Logs") {
            for (const XNode &m : e.kids) {
                if (m.name == "saveLogFiles") c.saveLogFiles = ival(&m) != 0;
                else if (m.name == "fetalID") c.fetalID = ival(&m);
                else if (m.name == "scale") c.scale = m.text;
                else if (m.name == "coordsystem") c.coordsystem = m.text;
                else if (m.name == "colormap") c.colormap = m.text;
                else if (m.name == "DetectionGrid") {
                    // ReadXML::ExtractLogsDetectionGrid (ReadXML.cpp:848-870): defaults 1
                    const char *keys[6] = {"x", "y", "z", "r", "phi", "rho"};
                    for (int k = 0; k < 6; ++k) c.detGrid[k] = fval(m.child(keys[k]), 1.0f);
                } else if (m.name == "filenames") {
                    for (const XNode &fn : m.kids) {
                        if (fn.name == "surface") c.surfaceFilename = fn.text;
                        else if (fn.name == "fetal") c.fetalFilename = fn.text;
                        else if (fn.name == "transmission") c.transmissionFilename = fn.text;
                        else if (fn.name == "absorbtionXZ") c.absorbXZFilename = fn.text;
                        else if (fn.name == "absorbtionYZ") c.absorbYZFilename = fn.text;
                    }
                }
            }
        }
    }
    c.modelfile = resolve(c.modelfile, cfgdir);
    c.emitterfile = resolve(c.emitterfile, cfgdir);
    if (c.tissues.empty()) throw std::runtime_error("config: no <tissueList>");
    return c;
}

Mesh ReadObj(const std::string &path, const std::vector<std::string> &names)
{
    std::ifstream f(path);
    if (!f) throw std::runtime_error("obj: cannot open " + path);
    std::vector<float> V, VN;
    Mesh m;
    int inner = 0, outer = 0;
    bool isSurface = false;
    std::string surfName, line, word;
    while (std::getline(f, line)) {
        if (!line.empty() && line.back() == '\r') line.pop_back();
        if (line.size() > 2 && line[0] == 'v' && line[1] == ' ') {
            std::istringstream is(line.substr(2));
            std::string a, b, c;
            is >> a >> b >> c;
            V.push_back(std::strtof(a.c_str(), nullptr));
            V.push_back(std::strtof(b.c_str(), nullptr));
            V.push_back(std::strtof(c.c_str(), nullptr));
            continue;
        }
        if (line.size() > 3 && line[0] == 'v' && line[1] == 'n' && line[2] == ' ') {
            std::istringstream is(line.substr(3));
            float a = 0, b = 0, c = 0;
            is >> a >> b >> c;
            VN.push_back(a);
            VN.push_back(b);
            VN.push_back(c);
            continue;
        }
        int gid = 0, gkind = 0;
        if (match_object(line, word)) {
            for (size_t i = 0; i < names.size(); ++i)
                if (word == names[i]) {
                    inner = (int)i;
                    break;
                }
        } else if (match_face(line)) {
            std::istringstream is(line.substr(2));
            std::string tok;
            std::vector<long> vi, ni;
            while (is >> tok) {
                long a = std::strtol(tok.c_str(), nullptr, 10);
                if (a < 0) a = (long)(V.size() / 3) + a + 1;  // relative indices
                vi.push_back(a - 1);
                size_t s2 = tok.rfind('/');
                ni.push_back(s2 != std::string::npos && tok.find('/') != s2 ? std::strtol(tok.c_str() + s2 + 1, nullptr, 10) - 1 : -1);
            }
            if (vi.size() < 3) throw std::runtime_error("obj: face with fewer than 3 vertices: " + line);
            for (int k = 0; k < 3; ++k) {
                if (vi[k] < 0 || vi[k] * 3 + 2 >= (long)V.size()) throw std::runtime_error("obj: bad vertex index: " + line);
                for (int a = 0; a < 3; ++a) m.tri.push_back(V[vi[k] * 3 + a]);
            }
            const float *A = &m.tri[m.tri.size() - 9], *B = A + 3, *Cc = A + 6;
            double e1[3], e2[3], n[3];
            for (int a = 0; a < 3; ++a) {
                e1[a] = (double)B[a] - A[a];
                e2[a] = (double)Cc[a] - A[a];
            }
            n[0] = e1[1] * e2[2] - e1[2] * e2[1];
            n[1] = e1[2] * e2[0] - e1[0] * e2[2];
            n[2] = e1[0] * e2[1] - e1[1] * e2[0];
            double l = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
            for (int a = 0; a < 3; ++a) m.nrm.push_back(l > 0 ? (float)(n[a] / l) : 0.0f);
            for (int a = 0; a < 3; ++a)
                m.vn.push_back((ni[0] >= 0 && ni[0] * 3 + 2 < (long)VN.size()) ? VN[ni[0] * 3 + a] : 0.0f);
            m.med.push_back(inner);
            m.med.push_back(outer);
            if (isSurface) {
                m.surface_ids.push_back((int32_t)(m.med.size() / 2 - 1));
                m.surface_names.push_back(surfName);
                surfName.clear();
            }
        } else if ((gkind = match_group(line, gid, word)) == 1) {
            isSurface = false;
            outer = gid;
        } else if (gkind == 2) {
            isSurface = true;
            outer = gid;
            surfName = word;
        }
    }
    if (m.tri.empty()) throw std::runtime_error("obj: no faces in " + path);
    return m;
}

void ReadEmitterFile(const std::string &path, std::vector<float> &angles, std::vector<float> &rri)
{
    // ImportExport::ImportEmitterModel (ImportExport.cpp:393-433)
    angles.clear();
    rri.clear();
    std::ifstream f(path);
    std::string line;
    float a = 0, b = 0;
    while (f && std::getline(f, line)) {
        if (!line.empty() && line.back() == '\r') line.pop_back();
        if (match_emitter_line(line, a, b)) {
            angles.push_back(a);
            rri.push_back(b);
        }
    }
    if (angles.empty()) {
        angles.push_back(0.0f);
        rri.push_back(1.0f);
    }
}

}  // namespace lp
