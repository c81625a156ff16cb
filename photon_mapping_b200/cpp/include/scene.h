// Drop-in for the reference's scene.h (scene.h:53-356): Scene with
// loadModel (OBJ + MTL, the reference loader's rules), build (upload and
// device BVH through pm_scene_upload) and intersect (pm_scene_intersect;
// the surface frame is filled on the host as scene.h:324-343 does).
#ifndef PM_DROPIN_SCENE_H
#define PM_DROPIN_SCENE_H
#include <cstdint>
#include <filesystem>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "core.h"
#include "photon_map.h"
#include "pm_cuda.h"
#include "primitive.h"
#include "spdlog/spdlog.h"

class Scene {
  std::vector<float> vertices;   // 9 per face (unshared, scene.h:199-212)
  std::vector<float> normals;    // 9 per face
  std::vector<float> texcoords;  // 6 per face
  std::vector<Vec3f> geometricNormals;
  std::vector<pm_material> materials;
  std::vector<Primitive> primitives;
  mutable pm_ctx* ctx = nullptr;

  struct Mtl {
    float kd[3] = {0, 0, 0}, ke[3] = {0, 0, 0}, ni = 1.0f;
    int illum = 0;
  };

  static std::map<std::string, Mtl> parseMtl(const std::filesystem::path& p) {
    std::map<std::string, Mtl> out;
    std::ifstream f(p);
    std::string line, cur;
    while (std::getline(f, line)) {
      std::istringstream ss(line);
      std::string tag;
      if (!(ss >> tag) || tag[0] == '#') continue;
      if (tag == "newmtl") {
        ss >> cur;
        out[cur] = Mtl();
      } else if (!cur.empty() && tag == "Kd") {
        ss >> out[cur].kd[0] >> out[cur].kd[1] >> out[cur].kd[2];
      } else if (!cur.empty() && tag == "Ke") {
        ss >> out[cur].ke[0] >> out[cur].ke[1] >> out[cur].ke[2];
      } else if (!cur.empty() && tag == "Ni") {
        ss >> out[cur].ni;
      } else if (!cur.empty() && tag == "illum") {
        ss >> out[cur].illum;
      }
    }
    return out;
  }

  void clear() {
    vertices.clear();
    normals.clear();
    texcoords.clear();
    geometricNormals.clear();
    materials.clear();
    primitives.clear();
  }

 public:
  Scene() {}
  Scene(const Scene&) = delete;
  Scene& operator=(const Scene&) = delete;
  ~Scene() {
    if (ctx) pm_ctx_destroy(ctx);
  }

  // scene.h:109-270. Polygons are fan-triangulated; MTL files are looked
  // up in the working directory (the reference's mtl_search_path "./").
  void loadModel(const std::filesystem::path& filepath) {
    clear();
    spdlog::info("[Scene] loading: {}", filepath.generic_string());
    std::ifstream f(filepath);
    if (!f) {
      spdlog::error("[Scene] failed to load {} : cannot open", filepath.generic_string());
      return;
    }
    std::vector<Vec3f> V, VN;
    std::vector<Vec2f> VT;
    std::map<std::string, Mtl> mtls;
    std::string line, cur;
    bool have_mtl = false;
    while (std::getline(f, line)) {
      std::istringstream ss(line);
      std::string tag;
      if (!(ss >> tag) || tag[0] == '#') continue;
      if (tag == "v") {
        float x, y, z;
        ss >> x >> y >> z;
        V.emplace_back(x, y, z);
      } else if (tag == "vn") {
        float x, y, z;
        ss >> x >> y >> z;
        VN.emplace_back(x, y, z);
      } else if (tag == "vt") {
        float x, y;
        ss >> x >> y;
        VT.emplace_back(x, y);
      } else if (tag == "mtllib") {
        std::string name;
        ss >> name;
        const auto m = parseMtl(std::filesystem::path("./") / name);
        mtls.insert(m.begin(), m.end());
      } else if (tag == "usemtl") {
        ss >> cur;
        have_mtl = true;
      } else if (tag == "f") {
        std::vector<int> vi, ti, ni;
        std::string c;
        while (ss >> c) {
          int idx[3] = {0, 0, 0};
          size_t pos = 0;
          for (int part = 0; part < 3; ++part) {
            const size_t slash = c.find('/', pos);
            const std::string tok = c.substr(pos, slash == std::string::npos ? std::string::npos
                                                                             : slash - pos);
            if (!tok.empty()) idx[part] = std::stoi(tok);
            if (slash == std::string::npos) break;
            pos = slash + 1;
          }
          auto fix = [](int i, size_t n) { return i > 0 ? i - 1 : (int)n + i; };
          vi.push_back(fix(idx[0], V.size()));
          ti.push_back(idx[1] ? fix(idx[1], VT.size()) : -1);
          ni.push_back(idx[2] ? fix(idx[2], VN.size()) : -1);
        }
        for (size_t t = 1; t + 1 < vi.size(); ++t) {
          const size_t corner[3] = {0, t, t + 1};
          Vec3f p[3], n[3];
          Vec2f uv[3];
          bool has_n = true, has_t = true;
          for (int k = 0; k < 3; ++k) {
            p[k] = V[vi[corner[k]]];
            if (ni[corner[k]] < 0) has_n = false; else n[k] = VN[ni[corner[k]]];
            if (ti[corner[k]] < 0) has_t = false; else uv[k] = VT[ti[corner[k]]];
          }
          if (!has_n) {  // scene.h:182-189
            const Vec3f e1 = normalize(p[1] - p[0]);
            const Vec3f e2 = normalize(p[2] - p[0]);
            n[0] = n[1] = n[2] = normalize(cross(e1, e2));
          }
          if (!has_t) {  // scene.h:192-196
            uv[0] = Vec2f(0, 0);
            uv[1] = Vec2f(1, 0);
            uv[2] = Vec2f(0, 1);
          }
          for (int k = 0; k < 3; ++k) {
            for (int a = 0; a < 3; ++a) {
              vertices.push_back(p[k][a]);
              normals.push_back(n[k][a]);
            }
            texcoords.push_back(uv[k][0]);
            texcoords.push_back(uv[k][1]);
          }
          // scene.h:15-51: illum 5 -> Mirror(1), 7 -> Glass(1, Ni), else
          // Lambert(Kd); Ke > 0 -> area light; no material -> Lambert(0.9)
          pm_material m{};
          m.type = PM_LAMBERT;
          m.rho[0] = m.rho[1] = m.rho[2] = 0.9f;
          m.ior = 1.0f;
          auto it = mtls.find(cur);
          if (have_mtl && it != mtls.end()) {
            const Mtl& mm = it->second;
            m.type = mm.illum == 5 ? PM_MIRROR : (mm.illum == 7 ? PM_GLASS : PM_LAMBERT);
            for (int a = 0; a < 3; ++a) {
              m.rho[a] = m.type == PM_LAMBERT ? mm.kd[a] : 1.0f;
              m.le[a] = mm.ke[a];
            }
            m.ior = mm.ni;
          }
          const uint32_t face = (uint32_t)materials.size();
          materials.push_back(m);
          geometricNormals.push_back(normalize(cross(p[1] - p[0], p[2] - p[0])));
          primitives.emplace_back(face, m);
        }
      }
    }
    spdlog::info("[Scene] vertices: {}", nVertices());
    spdlog::info("[Scene] faces: {}", nFaces());
  }

  uint32_t nVertices() const { return (uint32_t)(vertices.size() / 3); }
  uint32_t nFaces() const { return (uint32_t)(vertices.size() / 9); }
  pm_ctx* context() const { return ctx; }

  void build() {
    spdlog::info("[Scene] building scene...");
    if (!ctx)
      pm_dropin::check(nullptr, pm_ctx_create(pm_dropin::device_index(), &ctx), "pm_ctx_create");
    pm_dropin::check(ctx,
                     pm_scene_upload(ctx, vertices.data(), normals.data(), materials.data(),
                                     (int64_t)nFaces()),
                     "pm_scene_upload");
  }

  // scene.h:307-348
  bool intersect(const Ray& ray, IntersectInfo& info) const {
    const float r[8] = {ray.origin[0],    ray.origin[1],    ray.origin[2],    ray.tmin,
                        ray.direction[0], ray.direction[1], ray.direction[2], ray.tmax};
    pm_hit h;
    pm_dropin::check(ctx, pm_scene_intersect(ctx, r, 1, &h), "pm_scene_intersect");
    if (h.prim < 0) return false;
    info.t = h.t;
    SurfaceInfo& s = info.surfaceInfo;
    s.position = ray(info.t);
    s.barycentric = Vec2f(h.u, h.v);
    const size_t f = (size_t)h.prim;
    const float w0 = 1.0f - h.u - h.v;
    s.texcoords = Vec2f(texcoords[6 * f] * w0 + texcoords[6 * f + 2] * h.u + texcoords[6 * f + 4] * h.v,
                        texcoords[6 * f + 1] * w0 + texcoords[6 * f + 3] * h.u + texcoords[6 * f + 5] * h.v);
    s.geometricNormal = geometricNormals[f];
    const Vec3f n1(normals[9 * f], normals[9 * f + 1], normals[9 * f + 2]);
    const Vec3f n2(normals[9 * f + 3], normals[9 * f + 4], normals[9 * f + 5]);
    const Vec3f n3(normals[9 * f + 6], normals[9 * f + 7], normals[9 * f + 8]);
    s.shadingNormal = n1 * w0 + n2 * h.u + n3 * h.v;
    orthonormalBasis(s.shadingNormal, s.dpdu, s.dpdv);
    info.hitPrimitive = &primitives[f];
    return true;
  }
};

#endif
