// Reader of OpenParEM3D projects on the host: the .proj key/value file
// (project.c), the gmsh 2.2 ASCII mesh with physical volumes named after
// materials (mesh.cpp:449-588) or MFEM's ASCII mesh with the regions file
// materials_for_<mesh> (mesh.cpp:629-720), the ports file (Path / Port / Boundary blocks,
// port.cpp:6369-7078) and the materials databases (OpenParEMmaterials.cpp),
// turned into the inputs of opem_problem_create / set_regions / set_boundary /
// set_port_te.  Supported subset: ports on any planar closed path; a rectangle
// whose faces see one material is driven by its TE10 mode (the wide side is
// the mode's a dimension), every other port by the fundamental mode of its own
// faces (set_port_fem2d); the voltage integration path of the port's Line
// block sets the mode voltage; boundary
// types surface_impedance, perfect_electric_conductor, perfect_magnetic_conductor
// and radiation, frequency plans of point / linear / log entries (and their
// .refine forms).
// Exterior faces in no port or boundary path are PEC (the reference's default).
#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "engine.h"

namespace {

struct Mat { double er = 1, mur = 1, tand = 0, sigma = 0, Rz = 0; };
struct Path { std::vector<std::array<double, 3>> pts; bool closed = false; };
struct PortDef {
    std::string name, path, vpath, ipath, zdef = "PV";
    int sport = 0;
    int nmodes = 0;           // Line / Mode blocks (one per S-port of the port)
    bool composite = false;   // an integration path summed from several paths or scaled
};
struct BdrDef { std::string name, type, material; std::vector<std::string> paths; };

struct Project {
    std::string dir;
    std::map<std::string, std::vector<std::string>> kv;
    std::vector<double> verts;        // 3 per vertex
    std::vector<int64_t> tets;        // 4 per tet
    std::vector<int32_t> region;      // per tet
    std::vector<std::string> region_names;
    std::vector<Mat> region_mat;
    std::vector<int64_t> tris;        // exterior faces, 3 per face
    std::vector<int32_t> attr;        // per face
    std::vector<int64_t> tri_opp;     // vertex of the owning tet opposite the face
    std::vector<std::array<double, 22>> port_desc;
    std::vector<int> port_nsub;       // 0: analytic TE10; > 0: the port's own 2D mode on faces split nsub x nsub
    std::vector<int> port_zdef;       // OPEM_Z_PV / VI / PI
    std::vector<std::vector<double>> port_ipath;   // current path points (xyz)
    std::vector<int> port_ipath_closed;
    std::vector<std::pair<int, std::array<double, 3>>> bdr;   // attr -> (type, params)
    std::vector<double> freqs;
    int order = 1;
    int64_t n_port_faces = 0, n_bdr_faces = 0, n_pec_faces = 0;
};

std::string trim(const std::string& s) {
    size_t a = s.find_first_not_of(" \t\r\n"), b = s.find_last_not_of(" \t\r\n");
    return a == std::string::npos ? std::string() : s.substr(a, b - a + 1);
}

bool read_lines(const std::string& path, std::vector<std::string>& out) {
    std::ifstream f(path);
    if (!f) return false;
    std::string ln;
    while (std::getline(f, ln)) {
        const size_t c = ln.find("//");
        if (c != std::string::npos) ln = ln.substr(0, c);
        out.push_back(trim(ln));
    }
    return true;
}

std::string join(const std::string& dir, const std::string& f) {
    if (f.empty() || f[0] == '/') return f;
    return dir.empty() ? f : dir + "/" + f;
}

void parse_proj(const std::string& path, Project& P) {
    std::vector<std::string> L;
    if (!read_lines(path, L)) throw std::runtime_error("cannot read project file " + path);
    for (auto& ln : L) {
        if (ln.empty() || ln[0] == '#') continue;
        std::istringstream is(ln);
        std::string k, v;
        is >> k;
        std::getline(is, v);
        P.kv[k].push_back(trim(v));
    }
}

std::string kv1(const Project& P, const std::string& k, const std::string& dflt = "") {
    auto it = P.kv.find(k);
    return (it == P.kv.end() || it->second.empty()) ? dflt : it->second.back();
}

void read_gmsh22(const std::string& path, Project& P, std::vector<int>& phys) {
    std::ifstream f(path);
    if (!f) throw std::runtime_error("cannot read mesh " + path);
    std::string tok;
    std::map<int, std::string> names3;
    std::map<long, int64_t> idmap;
    while (f >> tok) {
        if (tok == "$PhysicalNames") {
            int n;
            f >> n;
            for (int i = 0; i < n; ++i) {
                int dim, tag;
                std::string name;
                f >> dim >> tag;
                std::getline(f, name);
                name = trim(name);
                if (name.size() >= 2 && name.front() == '"') name = name.substr(1, name.size() - 2);
                if (dim == 3) names3[tag] = name;
            }
        } else if (tok == "$Nodes") {
            long n;
            f >> n;
            for (long i = 0; i < n; ++i) {
                long id;
                double x, y, z;
                f >> id >> x >> y >> z;
                idmap[id] = (int64_t)P.verts.size() / 3;
                P.verts.insert(P.verts.end(), {x, y, z});
            }
        } else if (tok == "$Elements") {
            long n;
            f >> n;
            std::string line;
            std::getline(f, line);
            for (long i = 0; i < n; ++i) {
                std::getline(f, line);
                std::istringstream is(line);
                long id, type, ntags;
                is >> id >> type >> ntags;
                std::vector<long> tags(ntags);
                for (auto& t : tags) is >> t;
                if (type != 4) continue;   // only linear tetrahedra carry the volume
                long v[4];
                for (auto& x : v) is >> x;
                for (long x : v) {
                    auto it = idmap.find(x);
                    if (it == idmap.end()) throw std::runtime_error("element refers to an unknown node");
                    P.tets.push_back(it->second);
                }
                phys.push_back(ntags > 0 ? (int)tags[0] : 0);
            }
        }
    }
    if (P.tets.empty()) throw std::runtime_error("mesh has no tetrahedra");
    std::map<int, int> reg_of_tag;
    for (int t : phys)
        if (!reg_of_tag.count(t)) {
            reg_of_tag[t] = (int)P.region_names.size();
            auto it = names3.find(t);
            if (it == names3.end()) throw std::runtime_error("physical volume without a name (the name selects the material)");
            P.region_names.push_back(it->second);
        }
    for (int t : phys) P.region.push_back(reg_of_tag[t]);
}

// MFEM's ASCII mesh format (v1.0 / v1.2: "dimension", "elements" with attribute,
// geometry and vertex ids, "boundary", "vertices"), the other format the
// reference loads (MeshMaterialList::loadMFEM, src/OpenParEMCommon/mesh.cpp:629-720):
// the materials come from the regions file materials_for_<mesh file> beside it
// ("OpenParEM Regions v1.0", lines "index name"), element attribute a taking the
// name of index a - 1 (the material loop of OpenParEM3D.cpp:396-398).  Only the
// tetrahedra are read; the boundary is marked from the ports file, as for gmsh.
void read_mfem_mesh(const std::string& path, Project& P, std::vector<int>& phys) {
    std::ifstream f(path);
    if (!f) throw std::runtime_error("cannot read mesh " + path);
    std::string tok;
    std::getline(f, tok);
    int dim = 0;
    std::vector<std::array<int64_t, 4>> tets;
    while (f >> tok) {
        if (tok.empty() || tok[0] == '#') { std::getline(f, tok); continue; }
        if (tok == "dimension") {
            f >> dim;
        } else if (tok == "elements") {
            long n;
            f >> n;
            for (long i = 0; i < n; ++i) {
                int attr, geom;
                f >> attr >> geom;
                const int nv = geom == 4 ? 4 : (geom == 2 ? 3 : (geom == 5 ? 8 : (geom == 6 ? 6 : (geom == 7 ? 5 : (geom == 3 ? 4 : 2)))));
                std::array<int64_t, 8> v{};
                for (int k = 0; k < nv; ++k) f >> v[k];
                if (geom != 4) throw std::runtime_error("MFEM mesh: only tetrahedral volume elements are read");
                tets.push_back({v[0], v[1], v[2], v[3]});
                phys.push_back(attr);
            }
        } else if (tok == "boundary") {
            long n;
            f >> n;
            std::getline(f, tok);
            for (long i = 0; i < n; ++i) std::getline(f, tok);
        } else if (tok == "vertices") {
            long n;
            int vdim;
            f >> n >> vdim;
            if (vdim != 3) throw std::runtime_error("MFEM mesh: vertices must have 3 coordinates");
            for (long i = 0; i < n; ++i) {
                double x, y, z;
                f >> x >> y >> z;
                P.verts.insert(P.verts.end(), {x, y, z});
            }
            break;
        }
        if (!f) break;
    }
    if (dim != 3) throw std::runtime_error("MFEM mesh: dimension must be 3");
    if (tets.empty()) throw std::runtime_error("mesh has no tetrahedra");
    const int64_t nvt = (int64_t)P.verts.size() / 3;
    for (auto& t : tets)
        for (int64_t v : t) {
            if (v < 0 || v >= nvt) throw std::runtime_error("element refers to an unknown node");
            P.tets.push_back(v);
        }
    // the regions file
    const size_t sl = path.find_last_of('/');
    const std::string dir = sl == std::string::npos ? std::string() : path.substr(0, sl + 1);
    const std::string base = sl == std::string::npos ? path : path.substr(sl + 1);
    std::vector<std::string> L;
    if (!read_lines(dir + "materials_for_" + base, L) || L.empty() || L[0].rfind("OpenParEM Regions v", 0) != 0)
        throw std::runtime_error("MFEM mesh: regions file materials_for_" + base + " missing or malformed");
    std::map<int, std::string> names;
    for (size_t i = 1; i < L.size(); ++i) {
        std::string ln = trim(L[i].substr(0, L[i].find("//")));
        if (ln.empty()) continue;
        std::istringstream is(ln);
        int idx;
        std::string name;
        if (!(is >> idx >> name)) throw std::runtime_error("MFEM mesh: bad line in the regions file");
        if (name.size() >= 2 && name.front() == '"') name = name.substr(1, name.size() - 2);
        names[idx] = name;
    }
    std::map<int, int> reg_of_attr;
    for (int a : phys)
        if (!reg_of_attr.count(a)) {
            auto it = names.find(a - 1);
            if (it == names.end()) throw std::runtime_error("MFEM mesh: element attribute without a region name");
            reg_of_attr[a] = (int)P.region_names.size();
            P.region_names.push_back(it->second);
        }
    for (int a : phys) P.region.push_back(reg_of_attr[a]);
}

void read_materials(const std::string& path, std::map<std::string, Mat>& db) {
    std::vector<std::string> L;
    if (!read_lines(path, L)) return;   // a missing local database is not an error
    std::string name;
    Mat m;
    bool in_mat = false, have_freq = false, in_freq = false;
    for (auto& ln : L) {
        if (ln == "Material") { in_mat = true; name.clear(); m = Mat(); have_freq = false; continue; }
        if (ln == "EndMaterial") { if (in_mat && !name.empty()) db[name] = m; in_mat = false; continue; }
        if (!in_mat) continue;
        if (ln == "Frequency") { in_freq = !have_freq; continue; }   // the first frequency entry is used
        if (ln == "EndFrequency") { if (in_freq) have_freq = true; in_freq = false; continue; }
        const size_t e = ln.find('=');
        if (e == std::string::npos) continue;
        const std::string k = trim(ln.substr(0, e)), v = trim(ln.substr(e + 1));
        if (k == "name" && name.empty()) name = v;
        if (!in_freq) continue;
        if (k == "er") m.er = std::stod(v);
        else if (k == "mur") m.mur = std::stod(v);
        else if (k == "tand") m.tand = std::stod(v);
        else if (k == "conductivity") m.sigma = std::stod(v);
        else if (k == "Rz") m.Rz = std::stod(v);
    }
}

void read_ports(const std::string& path, std::map<std::string, Path>& paths, std::vector<PortDef>& ports,
                std::vector<BdrDef>& bdrs) {
    std::vector<std::string> L;
    if (!read_lines(path, L)) throw std::runtime_error("cannot read port definition file " + path);
    std::string block, pname, itype;
    bool in_ipath = false;
    Path cur;
    PortDef pd;
    BdrDef bd;
    for (auto& ln : L) {
        if (ln.empty() || ln[0] == '#') continue;
        if (ln == "Path" || ln == "Port" || ln == "Boundary" || ln == "File") {
            block = ln; cur = Path(); pname.clear(); pd = PortDef(); bd = BdrDef(); continue;
        }
        if (ln == "EndPath") { paths[pname] = cur; block.clear(); continue; }
        if (ln == "EndPort") {
            // ports with several conductors (several modes, composite integration
            // paths) need the multi-mode 2D solve, which is not built
            if (pd.nmodes > 1)
                throw std::runtime_error("port " + pd.name + " has " + std::to_string(pd.nmodes) +
                                         " modes: multi-conductor ports are not supported");
            if (pd.composite)
                throw std::runtime_error("port " + pd.name +
                                         ": integration paths summed from several paths or scaled are not supported");
            ports.push_back(pd);
            block.clear();
            continue;
        }
        if (block == "Port" && (ln == "Line" || ln == "Mode")) { ++pd.nmodes; continue; }
        if (ln == "EndBoundary") { bdrs.push_back(bd); block.clear(); continue; }
        if (ln == "EndFile") { block.clear(); continue; }
        if (ln == "IntegrationPath") { itype.clear(); in_ipath = true; continue; }
        if (ln == "EndIntegrationPath") { in_ipath = false; continue; }
        const size_t e = ln.find('=');
        if (e == std::string::npos) continue;
        const std::string k = trim(ln.substr(0, e)), v = trim(ln.substr(e + 1));
        if (block == "Path") {
            if (k == "name") pname = v;
            else if (k == "closed") cur.closed = (v == "true");
            else if (k == "point") {
                std::string s = v;
                for (char& c : s) if (c == '(' || c == ')' || c == ',') c = ' ';
                std::istringstream is(s);
                std::array<double, 3> p{};
                is >> p[0] >> p[1] >> p[2];
                cur.pts.push_back(p);
            }
        } else if (block == "Port") {
            if (in_ipath) {
                if (k == "type") itype = v;
                else if (k == "path+" || k == "path-" || k == "scale") pd.composite = true;
                else if (k == "path" && itype == "voltage" && pd.vpath.empty()) pd.vpath = v;
                else if (k == "path" && itype == "current" && pd.ipath.empty()) pd.ipath = v;
            } else if (k == "name") {
                pd.name = v;
            } else if (k == "path") {
                pd.path = v;
            } else if (k == "Sport") {
                pd.sport = std::stoi(v);
            } else if (k == "impedance_definition") {
                pd.zdef = v;
            }
        } else if (block == "Boundary") {
            if (k == "name") bd.name = v;
            else if (k == "type") bd.type = v;
            else if (k == "material") bd.material = v;
            else if (k == "path") bd.paths.push_back(v);
        }
    }
}

// signed path reference "+name" / "-name" -> points (reversed for "-")
std::vector<std::array<double, 3>> path_points(const std::map<std::string, Path>& paths, const std::string& ref,
                                               bool* closed = nullptr) {
    std::string nm = ref;
    bool rev = false;
    if (!nm.empty() && (nm[0] == '+' || nm[0] == '-')) { rev = nm[0] == '-'; nm = nm.substr(1); }
    auto it = paths.find(nm);
    if (it == paths.end()) throw std::runtime_error("unknown path " + nm);
    auto pts = it->second.pts;
    if (rev) std::reverse(pts.begin(), pts.end());
    if (closed) *closed = it->second.closed;
    return pts;
}

using V3 = std::array<double, 3>;
V3 sub(const V3& a, const V3& b) { return {a[0] - b[0], a[1] - b[1], a[2] - b[2]}; }
double dot(const V3& a, const V3& b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
V3 cross(const V3& a, const V3& b) { return {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]}; }
double norm(const V3& a) { return std::sqrt(dot(a, a)); }
V3 scale(const V3& a, double s) { return {a[0] * s, a[1] * s, a[2] * s}; }

// planar closed polygon: does point x lie in its plane and inside (edges included)?
struct Poly {
    V3 o, n, u, v;
    std::vector<std::array<double, 2>> q;
    double tol;
    explicit Poly(const std::vector<V3>& pts, double tol_) : tol(tol_) {
        if (pts.size() < 3) throw std::runtime_error("a closed path needs at least three points");
        o = pts[0];
        n = {0.0, 0.0, 0.0};
        for (size_t i = 1; i + 1 < pts.size() && norm(n) < 1e-30; ++i) n = cross(sub(pts[i], o), sub(pts[i + 1], o));
        if (!(norm(n) > 0)) throw std::runtime_error("degenerate closed path");
        n = scale(n, 1.0 / norm(n));
        u = sub(pts[1], o);
        u = scale(u, 1.0 / norm(u));
        v = cross(n, u);
        for (auto& p : pts) q.push_back({dot(sub(p, o), u), dot(sub(p, o), v)});
    }
    bool contains(const V3& x) const {
        const V3 d = sub(x, o);
        if (std::fabs(dot(d, n)) > tol) return false;
        const double px = dot(d, u), py = dot(d, v);
        const size_t m = q.size();
        for (size_t i = 0; i < m; ++i) {   // on an edge (within tol)?
            const auto& a = q[i];
            const auto& b = q[(i + 1) % m];
            const double ex = b[0] - a[0], ey = b[1] - a[1], L2 = ex * ex + ey * ey;
            const double t = L2 > 0 ? std::max(0.0, std::min(1.0, ((px - a[0]) * ex + (py - a[1]) * ey) / L2)) : 0;
            const double dx = a[0] + t * ex - px, dy = a[1] + t * ey - py;
            if (dx * dx + dy * dy <= tol * tol) return true;
        }
        bool in = false;   // crossing test
        for (size_t i = 0, j = m - 1; i < m; j = i++) {
            const auto& a = q[i];
            const auto& b = q[j];
            if (((a[1] > py) != (b[1] > py)) && (px < (b[0] - a[0]) * (py - a[1]) / (b[1] - a[1]) + a[0])) in = !in;
        }
        return in;
    }
};

// four corners with right angles (within tol of the longer side)
bool is_rectangle(const std::vector<V3>& pts, double tol) {
    if (pts.size() != 4) return false;
    for (int i = 0; i < 4; ++i) {
        const V3 e1 = sub(pts[(i + 1) % 4], pts[i]), e2 = sub(pts[(i + 3) % 4], pts[i]);
        const double l1 = norm(e1), l2 = norm(e2);
        if (!(l1 > 0 && l2 > 0)) return false;
        if (std::fabs(dot(e1, e2)) > tol * std::max(l1, l2)) return false;
    }
    return true;
}

void build(const std::string& proj_path, int order_override, Project& P) {
    const size_t sl = proj_path.find_last_of('/');
    P.dir = sl == std::string::npos ? std::string() : proj_path.substr(0, sl);
    parse_proj(proj_path, P);
    const std::string mesh = kv1(P, "mesh.file");
    if (mesh.empty()) throw std::runtime_error("project names no mesh.file");
    P.order = std::atoi(kv1(P, "mesh.order", "1").c_str());
    if (order_override > 0) P.order = order_override;
    std::vector<int> phys;
    {
        std::ifstream probe(join(P.dir, mesh));
        std::string first;
        std::getline(probe, first);
        first = trim(first);
        if (first == "MFEM mesh v1.0" || first == "MFEM mesh v1.2") read_mfem_mesh(join(P.dir, mesh), P, phys);
        else read_gmsh22(join(P.dir, mesh), P, phys);
    }
    // materials: global database, then the local one overrides
    std::map<std::string, Mat> db;
    read_materials(join(join(P.dir, kv1(P, "materials.global.path")), kv1(P, "materials.global.name")), db);
    read_materials(join(join(P.dir, kv1(P, "materials.local.path")), kv1(P, "materials.local.name")), db);
    for (auto& nm : P.region_names) {
        auto it = db.find(nm);
        if (it == db.end()) throw std::runtime_error("material " + nm + " not in the materials databases");
        P.region_mat.push_back(it->second);
    }
    // frequency plan
    for (auto k : {"frequency.plan.point", "frequency.plan.point.refine"}) {
        auto it = P.kv.find(k);
        if (it != P.kv.end())
            for (auto& v : it->second) P.freqs.push_back(std::stod(v));
    }
    // linear plans: start, stop, step, the step added repeatedly; log plans: start,
    // stop, points per decade, the factor 10^(1/points) applied repeatedly; both up
    // to stop (1 + 1e-12) (FrequencyPlan, OpenParEMCommon/frequencyPlan.cpp:137-197;
    // the .refine forms give the same points)
    for (auto k : {"frequency.plan.linear", "frequency.plan.linear.refine", "frequency.plan.log",
                   "frequency.plan.log.refine"}) {
        auto it = P.kv.find(k);
        if (it == P.kv.end()) continue;
        const bool lg = std::string(k).find(".log") != std::string::npos;
        for (auto v : it->second) {
            v = v.substr(0, v.find("//"));
            for (char& c : v) if (c == ',') c = ' ';
            std::istringstream is(v);
            double a = 0, b = 0, st = 0;
            std::string third, extra;
            if (!(is >> a >> b >> third) || (is >> extra) || !(a > 0)) throw std::runtime_error(std::string("bad ") + k);
            if (lg) {
                // points per decade is an integer (project.c reads it with is_int/atoi)
                size_t q = (third[0] == '+') ? 1 : 0;
                if (q == third.size() || third.find_first_not_of("0123456789", q) != std::string::npos)
                    throw std::runtime_error(std::string("bad ") + k + ": points per decade must be an integer");
                st = std::atof(third.c_str());
            } else {
                char* end = nullptr;
                st = std::strtod(third.c_str(), &end);
                if (!end || *end) throw std::runtime_error(std::string("bad ") + k);
            }
            if (!(st > 0)) throw std::runtime_error(std::string("bad ") + k);
            const double factor = lg ? std::pow(10.0, 1.0 / st) : 0.0;
            for (double f = a; f <= b * (1 + 1e-12); f = lg ? f * factor : f + st) {
                P.freqs.push_back(f);
                if (P.freqs.size() > 10000000) throw std::runtime_error(std::string("too many points in ") + k);
            }
        }
    }
    // duplicates: relative difference below 1e-14 (FrequencyPlan::eliminateDuplicates,
    // OpenParEMCommon/frequencyPlan.cpp:60-84)
    std::sort(P.freqs.begin(), P.freqs.end());
    P.freqs.erase(std::unique(P.freqs.begin(), P.freqs.end(),
                              [](double x, double y) { return std::fabs(y - x) < 1e-14 * std::fabs(y); }),
                  P.freqs.end());
    // exterior faces with the opposite vertex of their tet
    const int64_t ne = (int64_t)P.tets.size() / 4;
    struct FaceUse { int count = 0; int64_t second = -1, tet = -1; };   // uses, opposite vertex, owning tet
    std::map<std::array<int64_t, 3>, FaceUse> faces;
    static const int F[4][4] = {{1, 2, 3, 0}, {0, 2, 3, 1}, {0, 1, 3, 2}, {0, 1, 2, 3}};
    for (int64_t e = 0; e < ne; ++e)
        for (auto& f : F) {
            std::array<int64_t, 3> k = {P.tets[4 * e + f[0]], P.tets[4 * e + f[1]], P.tets[4 * e + f[2]]};
            std::sort(k.begin(), k.end());
            auto& c = faces[k];
            c.count += 1;
            c.second = P.tets[4 * e + f[3]];
            c.tet = e;
        }
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (size_t i = 0; i < P.verts.size(); ++i) {
        lo[i % 3] = std::min(lo[i % 3], P.verts[i]);
        hi[i % 3] = std::max(hi[i % 3], P.verts[i]);
    }
    const double tol = 1e-6 * std::max({hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]});
    std::map<std::string, Path> paths;
    std::vector<PortDef> ports;
    std::vector<BdrDef> bdrs;
    read_ports(join(P.dir, kv1(P, "port.definition.file")), paths, ports, bdrs);
    std::sort(ports.begin(), ports.end(), [](const PortDef& a, const PortDef& b) { return a.sport < b.sport; });
    std::vector<Poly> port_poly;
    std::vector<int> port_rect;   // 1: a rectangle (driven by TE10 where its faces see one material)
    for (auto& pd : ports) {
        bool closed = false;
        auto pts = path_points(paths, pd.path, &closed);
        if (!closed) throw std::runtime_error("port " + pd.name + ": the port path must be closed");
        port_poly.emplace_back(pts, tol);
        port_rect.push_back(is_rectangle(pts, tol) ? 1 : 0);
    }
    std::vector<std::vector<Poly>> bdr_poly(bdrs.size());
    for (size_t j = 0; j < bdrs.size(); ++j)
        for (auto& r : bdrs[j].paths) bdr_poly[j].emplace_back(path_points(paths, r), tol);
    auto vtx = [&](int64_t i) { return V3{P.verts[3 * i], P.verts[3 * i + 1], P.verts[3 * i + 2]}; };
    const int np = (int)ports.size(), nb = (int)bdrs.size();
    std::vector<int64_t> port_opp(np, -1), port_face0(np, -1), port_nface(np, 0);
    std::vector<int> port_mixed(np, 0), port_reg0(np, -1);   // faces of more than one material behind the port
    std::vector<double> port_area(np, 0.0);                  // area of the port's faces
    auto same_mat = [&](int r0, int r1) {
        const Mat &A = P.region_mat[r0], &B = P.region_mat[r1];
        return A.er == B.er && A.tand == B.tand && A.sigma == B.sigma && A.mur == B.mur;
    };
    for (auto& kvf : faces) {
        if (kvf.second.count != 1) continue;
        const auto& k = kvf.first;
        int a = 1;   // PEC
        for (int p = 0; p < np && a == 1; ++p)
            if (port_poly[p].contains(vtx(k[0])) && port_poly[p].contains(vtx(k[1])) && port_poly[p].contains(vtx(k[2]))) {
                a = 2 + p;
                if (port_opp[p] < 0) { port_opp[p] = kvf.second.second; port_face0[p] = k[0]; }
                const int r = P.region[kvf.second.tet];
                if (port_reg0[p] < 0) port_reg0[p] = r;
                else if (!same_mat(port_reg0[p], r)) port_mixed[p] = 1;
                ++port_nface[p];
                port_area[p] += 0.5 * norm(cross(sub(vtx(k[1]), vtx(k[0])), sub(vtx(k[2]), vtx(k[0]))));
            }
        for (int j = 0; j < nb && a == 1; ++j)
            for (auto& poly : bdr_poly[j])
                if (poly.contains(vtx(k[0])) && poly.contains(vtx(k[1])) && poly.contains(vtx(k[2]))) { a = 2 + np + j; break; }
        P.tris.insert(P.tris.end(), k.begin(), k.end());
        P.attr.push_back(a);
        if (a == 1) ++P.n_pec_faces;
        else if (a < 2 + np) ++P.n_port_faces;
        else ++P.n_bdr_faces;
    }
    // port frames: on a rectangle TE10's, a along the wide side; on any other
    // polygon u along its first edge, v in its plane, a x b its bounding box
    // in (u, v); outward normal
    for (int p = 0; p < np; ++p) {
        if (port_opp[p] < 0) throw std::runtime_error("port " + ports[p].name + " covers no boundary face");
        auto pts = path_points(paths, ports[p].path);
        V3 o = pts[0], u, v;
        double a, b;
        if (port_rect[p]) {
            V3 e1 = sub(pts[1], pts[0]), e2 = sub(pts[3], pts[0]);
            if (norm(e2) > norm(e1)) std::swap(e1, e2);
            a = norm(e1);
            b = norm(e2);
            u = scale(e1, 1.0 / a);
            v = scale(e2, 1.0 / b);
        } else {
            const Poly& pg = port_poly[p];
            u = pg.u;
            v = pg.v;
            double lo_u = 1e300, hi_u = -1e300, lo_v = 1e300, hi_v = -1e300;
            for (auto& q : pg.q) {
                lo_u = std::min(lo_u, q[0]); hi_u = std::max(hi_u, q[0]);
                lo_v = std::min(lo_v, q[1]); hi_v = std::max(hi_v, q[1]);
            }
            for (int i = 0; i < 3; ++i) o[i] = pg.o[i] + lo_u * u[i] + lo_v * v[i];   // bounding-box corner
            a = hi_u - lo_u;
            b = hi_v - lo_v;
        }
        V3 n = cross(u, v);
        if (dot(sub(vtx(port_opp[p]), vtx(port_face0[p])), n) > 0) n = scale(n, -1.0);   // point out of the mesh
        std::array<double, 22> d{};
        for (int i = 0; i < 3; ++i) { d[i] = o[i]; d[3 + i] = u[i]; d[6 + i] = v[i]; d[9 + i] = n[i]; }
        d[12] = a; d[13] = b; d[14] = 1; d[15] = 0;
        // default voltage path: across the narrow side at the middle of the wide one
        V3 vs = {o[0] + 0.5 * a * u[0], o[1] + 0.5 * a * u[1], o[2] + 0.5 * a * u[2]};
        V3 ve = {vs[0] + b * v[0], vs[1] + b * v[1], vs[2] + b * v[2]};
        if (!ports[p].vpath.empty()) {
            auto vp = path_points(paths, ports[p].vpath);
            vs = vp.front();
            ve = vp.back();
        }
        for (int i = 0; i < 3; ++i) { d[16 + i] = vs[i]; d[19 + i] = ve[i]; }
        P.port_desc.push_back(d);
        // a port whose faces see more than one material is driven by its own 2D
        // mode (as the reference drives every port), solved as the reference's 2D
        // solver does: on the port faces themselves (no split) with elements of the
        // problem's order, so the mode lies in the 3D port trace space
        // (and every port that is not a rectangle, which has no analytic mode here)
        const int nsub = 1;
        // faces that leave part of the port polygon uncovered (a conductor inside
        // the cross-section is a hole in them): no analytic mode either
        double parea = 0.0;
        {
            const auto& q = port_poly[p].q;
            for (size_t i = 0; i < q.size(); ++i) {
                const auto& a0 = q[i];
                const auto& a1 = q[(i + 1) % q.size()];
                parea += 0.5 * (a0[0] * a1[1] - a1[0] * a0[1]);
            }
            parea = std::fabs(parea);
        }
        const bool holes = port_area[p] < (1.0 - 1e-9) * parea;
        // impedance definition and current path (a port that uses its current
        // is driven by its own 2D mode, where the current is integrated)
        const std::string& zd = ports[p].zdef;
        int zdef = OPEM_Z_PV;
        if (zd == "VI") zdef = OPEM_Z_VI;
        else if (zd == "PI") zdef = OPEM_Z_PI;
        else if (zd != "PV") throw std::runtime_error("port " + ports[p].name + ": impedance_definition must be VI, PV or PI");
        std::vector<double> ip;
        int ipc = 1;
        if (!ports[p].ipath.empty()) {
            bool cl = false;
            for (auto& q : path_points(paths, ports[p].ipath, &cl)) ip.insert(ip.end(), q.begin(), q.end());
            ipc = cl ? 1 : 0;
        }
        if (zdef != OPEM_Z_PV && ip.size() < 6)
            throw std::runtime_error("port " + ports[p].name + ": impedance_definition " + zd + " needs a current path");
        P.port_zdef.push_back(zdef);
        P.port_ipath.push_back(ip);
        P.port_ipath_closed.push_back(ipc);
        P.port_nsub.push_back(port_mixed[p] || !port_rect[p] || holes || zdef != OPEM_Z_PV ? nsub : 0);
    }
    // boundary conditions: attribute 1 the faces no port or Boundary block claims
    // (PEC, or the surface impedance of materials.default.boundary, as
    // BoundaryDatabase::createDefaultBoundary does, port.cpp:7047-7078), ports
    // 2.., the Boundary blocks after them
    std::string dflt = kv1(P, "materials.default.boundary", "PEC");
    dflt = trim(dflt.substr(0, dflt.find("//")));
    if (dflt.empty()) dflt = "PEC";
    if (dflt == "PEC") {
        P.bdr.push_back({OPEM_BDR_PEC, {0, 0, 0}});
    } else {
        auto it = db.find(dflt);
        if (it == db.end()) throw std::runtime_error("default boundary material " + dflt + " not found");
        P.bdr.push_back({OPEM_BDR_IMPEDANCE, {it->second.sigma, it->second.Rz, it->second.mur}});
        P.n_bdr_faces += P.n_pec_faces;
        P.n_pec_faces = 0;
    }
    for (int p = 0; p < np; ++p) P.bdr.push_back({OPEM_BDR_PORT, {(double)p, 0, 0}});
    for (auto& bd : bdrs) {
        if (bd.type == "surface_impedance") {
            auto it = db.find(bd.material);
            if (it == db.end()) throw std::runtime_error("boundary material " + bd.material + " not found");
            P.bdr.push_back({OPEM_BDR_IMPEDANCE, {it->second.sigma, it->second.Rz, it->second.mur}});
        } else if (bd.type == "perfect_electric_conductor") {
            P.bdr.push_back({OPEM_BDR_PEC, {0, 0, 0}});
        } else if (bd.type == "perfect_magnetic_conductor") {
            P.bdr.push_back({OPEM_BDR_PMC, {0, 0, 0}});
        } else if (bd.type == "radiation") {
            P.bdr.push_back({OPEM_BDR_RADIATION, {std::sqrt(4e-7 * M_PI / 8.8541878176e-12), 0, 0}});
        } else {
            throw std::runtime_error("boundary type " + bd.type + " is not supported");
        }
    }
}

}  // namespace

extern "C" {

int opem_project_value(const char* proj_path, const char* key, char* buf, int len) {
    if (!proj_path || !key || !buf || len < 1) return OPEM_ERR_ARG;
    buf[0] = 0;
    Project P;
    try {
        parse_proj(proj_path, P);
    } catch (const std::exception&) {
        return OPEM_ERR_ARG;
    }
    auto it = P.kv.find(key);
    if (it == P.kv.end() || it->second.empty()) return OPEM_ERR_ARG;
    const std::string v = trim(it->second.back().substr(0, it->second.back().find("//")));
    if ((int)v.size() >= len) return OPEM_ERR_ARG;
    std::memcpy(buf, v.c_str(), v.size() + 1);
    return OPEM_OK;
}

int opem_project_info(const char* proj_path, int order, int64_t* info, int ninfo, double* freqs, int max_freqs,
                      char* msg, int msg_len) {
    if (!proj_path || !info) return OPEM_ERR_ARG;
    Project P;
    try {
        build(proj_path, order, P);
    } catch (const std::exception& e) {
        if (msg && msg_len > 0) { std::strncpy(msg, e.what(), msg_len - 1); msg[msg_len - 1] = 0; }
        return OPEM_ERR_ARG;
    }
    const int64_t v[10] = {(int64_t)P.verts.size() / 3, (int64_t)P.tets.size() / 4, (int64_t)P.region_names.size(),
                           (int64_t)P.attr.size(), P.n_port_faces, P.n_bdr_faces, P.n_pec_faces,
                           (int64_t)P.port_desc.size(), (int64_t)P.freqs.size(), P.order};
    for (int i = 0; i < ninfo && i < 10; ++i) info[i] = v[i];
    if (freqs)
        for (int i = 0; i < max_freqs && i < (int)P.freqs.size(); ++i) freqs[i] = P.freqs[i];
    if (msg && msg_len > 0) msg[0] = 0;
    return OPEM_OK;
}

int opem_project_read(const char* proj_path, int order, int64_t* counts, double* verts, int64_t* tets,
                      int32_t* region, double* region_mat, int64_t* tris, int32_t* attr, int32_t* bdr_type,
                      double* bdr_params, double* port_desc, int32_t* port_nsub, double* freqs, char* msg,
                      int msg_len) {
    if (!proj_path || !counts) return OPEM_ERR_ARG;
    Project P;
    try {
        build(proj_path, order, P);
    } catch (const std::exception& e) {
        if (msg && msg_len > 0) { std::strncpy(msg, e.what(), msg_len - 1); msg[msg_len - 1] = 0; }
        return OPEM_ERR_ARG;
    }
    const int64_t nv = (int64_t)P.verts.size() / 3, ne = (int64_t)P.tets.size() / 4, nr = (int64_t)P.region_mat.size();
    const int64_t nf = (int64_t)P.attr.size(), na = (int64_t)P.bdr.size(), np = (int64_t)P.port_desc.size();
    const int64_t nq = (int64_t)P.freqs.size();
    counts[0] = nv; counts[1] = ne; counts[2] = nr; counts[3] = nf; counts[4] = na; counts[5] = np; counts[6] = nq;
    counts[7] = P.order;
    if (verts) std::memcpy(verts, P.verts.data(), P.verts.size() * sizeof(double));
    if (tets) std::memcpy(tets, P.tets.data(), P.tets.size() * sizeof(int64_t));
    if (region) std::memcpy(region, P.region.data(), P.region.size() * sizeof(int32_t));
    if (region_mat)
        for (int64_t r = 0; r < nr; ++r) {
            region_mat[4 * r + 0] = P.region_mat[r].er;
            region_mat[4 * r + 1] = P.region_mat[r].tand;
            region_mat[4 * r + 2] = P.region_mat[r].sigma;
            region_mat[4 * r + 3] = P.region_mat[r].mur;
        }
    if (tris) std::memcpy(tris, P.tris.data(), P.tris.size() * sizeof(int64_t));
    if (attr) std::memcpy(attr, P.attr.data(), P.attr.size() * sizeof(int32_t));
    for (int64_t a = 0; a < na; ++a) {
        if (bdr_type) bdr_type[a] = P.bdr[a].first;
        if (bdr_params)
            for (int i = 0; i < 3; ++i) bdr_params[3 * a + i] = P.bdr[a].second[i];
    }
    if (port_desc)
        for (int64_t p = 0; p < np; ++p)
            for (int i = 0; i < 22; ++i) port_desc[22 * p + i] = P.port_desc[p][i];
    if (port_nsub)
        for (int64_t p = 0; p < np; ++p) port_nsub[p] = P.port_nsub[p];
    if (freqs)
        for (int64_t q = 0; q < nq; ++q) freqs[q] = P.freqs[q];
    if (msg && msg_len > 0) msg[0] = 0;
    return OPEM_OK;
}

int opem_project_port_impedance(const char* proj_path, int port, int* definition, int* closed, int* npath,
                                double* path, int cap, char* msg, int msg_len) {
    if (!proj_path || port < 0 || !definition || !closed || !npath || cap < 0 || (cap > 0 && !path))
        return OPEM_ERR_ARG;
    Project P;
    try {
        build(proj_path, 0, P);
    } catch (const std::exception& e) {
        if (msg && msg_len > 0) { std::strncpy(msg, e.what(), msg_len - 1); msg[msg_len - 1] = 0; }
        return OPEM_ERR_ARG;
    }
    if (port >= (int)P.port_zdef.size()) return OPEM_ERR_ARG;
    *definition = P.port_zdef[port];
    *closed = P.port_ipath_closed[port];
    *npath = (int)(P.port_ipath[port].size() / 3);
    for (int i = 0; i < 3 * std::min(cap, *npath); ++i) path[i] = P.port_ipath[port][i];
    return OPEM_OK;
}

int opem_project_load(opem_context ctx, const char* proj_path, int order, opem_problem* out, int* nfreq,
                      double* freqs, int max_freqs) {
    if (!ctx || !proj_path || !out) return OPEM_ERR_ARG;
    *out = nullptr;
    Project P;
    try {
        build(proj_path, order, P);
    } catch (const std::exception& e) {
        ctx->c.last_error = std::string("opem_project_load: ") + e.what();
        return OPEM_ERR_ARG;
    }
    if (P.order < 1 || P.order > 3) {
        ctx->c.last_error = "opem_project_load: mesh.order " + std::to_string(P.order) + " (orders 1-3 are built; pass order)";
        return OPEM_ERR_UNSUPPORTED;
    }
    opem_problem prob = nullptr;
    int rc = opem_problem_create(ctx, (int64_t)P.verts.size() / 3, P.verts.data(), (int64_t)P.tets.size() / 4,
                                 P.tets.data(), P.region.data(), (int64_t)P.attr.size(), P.tris.data(), P.attr.data(),
                                 P.order, &prob);
    if (rc != OPEM_OK) return rc;
    const int nr = (int)P.region_mat.size();
    std::vector<double> er(nr), td(nr), sg(nr), mr(nr);
    for (int r = 0; r < nr; ++r) {
        er[r] = P.region_mat[r].er; td[r] = P.region_mat[r].tand; sg[r] = P.region_mat[r].sigma; mr[r] = P.region_mat[r].mur;
    }
    rc = opem_problem_set_regions(prob, nr, er.data(), td.data(), sg.data(), mr.data());
    for (size_t a = 0; rc == OPEM_OK && a < P.bdr.size(); ++a) {
        const int type = P.bdr[a].first;
        const int np = type == OPEM_BDR_PORT ? 1 : (type == OPEM_BDR_IMPEDANCE ? 3 : (type == OPEM_BDR_RADIATION ? 1 : 0));
        rc = opem_problem_set_boundary(prob, (int)a + 1, type, np ? P.bdr[a].second.data() : nullptr, np);
    }
    for (size_t p = 0; rc == OPEM_OK && p < P.port_desc.size(); ++p) {
        rc = P.port_nsub[p] > 0 ? opem_problem_set_port_fem2d(prob, (int)p, P.port_desc[p].data(), P.port_nsub[p],
                                                              std::min(8, P.order))
                                : opem_problem_set_port_te(prob, (int)p, P.port_desc[p].data());
        if (rc == OPEM_OK && P.port_nsub[p] > 0 && !P.port_ipath[p].empty())
            rc = opem_problem_set_port_impedance(prob, (int)p, P.port_zdef[p], (int)(P.port_ipath[p].size() / 3),
                                                 P.port_ipath[p].data(), P.port_ipath_closed[p]);
    }
    if (rc != OPEM_OK) {
        opem_problem_destroy(prob);
        return rc;
    }
    if (nfreq) *nfreq = (int)P.freqs.size();
    if (freqs)
        for (int i = 0; i < max_freqs && i < (int)P.freqs.size(); ++i) freqs[i] = P.freqs[i];
    *out = prob;
    return OPEM_OK;
}

}  // extern "C"

