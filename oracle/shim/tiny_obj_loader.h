// ORACLE shim — test infrastructure only. A project-written stand-in for
// the part of the tinyobjloader API that the reference's scene.h calls
// (scene.h:21-51, 114-133, 215): ObjReader::ParseFromFile with
// triangulation (polygons split as a fan) and MTL loading from
// mtl_search_path; attrib/shape/material records with the members scene.h
// reads. tinyobjloader's own source is not used or reproduced.
#pragma once
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

namespace tinyobj {
typedef float real_t;
struct index_t {
  int vertex_index, normal_index, texcoord_index;
};
struct mesh_t {
  std::vector<index_t> indices;
  std::vector<unsigned char> num_face_vertices;
  std::vector<int> material_ids;
};
struct shape_t {
  std::string name;
  mesh_t mesh;
};
struct attrib_t {
  std::vector<real_t> vertices, normals, texcoords;
};
struct material_t {
  std::string name;
  real_t ambient[3] = {0, 0, 0}, diffuse[3] = {0, 0, 0}, specular[3] = {0, 0, 0};
  real_t transmittance[3] = {0, 0, 0}, emission[3] = {0, 0, 0};
  real_t shininess = 1, ior = 1, dissolve = 1;
  int illum = 0;
};
struct ObjReaderConfig {
  bool triangulate = true;
  std::string mtl_search_path;
};

class ObjReader {
  attrib_t attrib_;
  std::vector<shape_t> shapes_;
  std::vector<material_t> materials_;
  std::string warning_, error_;

  void load_mtl(const std::string& path, std::map<std::string, int>& ids) {
    std::ifstream f(path);
    if (!f) {
      warning_ += "material file not found: " + path + "\n";
      return;
    }
    std::string line;
    while (std::getline(f, line)) {
      std::istringstream ss(line);
      std::string tag;
      if (!(ss >> tag) || tag[0] == '#') continue;
      if (tag == "newmtl") {
        material_t m;
        ss >> m.name;
        ids[m.name] = (int)materials_.size();
        materials_.push_back(m);
      } else if (materials_.empty()) {
        continue;
      } else if (tag == "Ka") {
        ss >> materials_.back().ambient[0] >> materials_.back().ambient[1] >> materials_.back().ambient[2];
      } else if (tag == "Kd") {
        ss >> materials_.back().diffuse[0] >> materials_.back().diffuse[1] >> materials_.back().diffuse[2];
      } else if (tag == "Ks") {
        ss >> materials_.back().specular[0] >> materials_.back().specular[1] >> materials_.back().specular[2];
      } else if (tag == "Ke") {
        ss >> materials_.back().emission[0] >> materials_.back().emission[1] >> materials_.back().emission[2];
      } else if (tag == "Ni") {
        ss >> materials_.back().ior;
      } else if (tag == "Ns") {
        ss >> materials_.back().shininess;
      } else if (tag == "d") {
        ss >> materials_.back().dissolve;
      } else if (tag == "illum") {
        ss >> materials_.back().illum;
      }
    }
  }

 public:
  bool ParseFromFile(const std::string& filename, const ObjReaderConfig& config = ObjReaderConfig()) {
    std::ifstream f(filename);
    if (!f) {
      error_ = "cannot open " + filename;
      return false;
    }
    shapes_.assign(1, shape_t());
    std::map<std::string, int> ids;
    int cur = -1;
    std::string line;
    auto fix = [](int i, size_t n) { return i > 0 ? i - 1 : (int)n / 3 + i; };
    while (std::getline(f, line)) {
      std::istringstream ss(line);
      std::string tag;
      if (!(ss >> tag) || tag[0] == '#') continue;
      if (tag == "v" || tag == "vn") {
        real_t x, y, z;
        ss >> x >> y >> z;
        auto& dst = tag == "v" ? attrib_.vertices : attrib_.normals;
        dst.push_back(x);
        dst.push_back(y);
        dst.push_back(z);
      } else if (tag == "vt") {
        real_t x, y;
        ss >> x >> y;
        attrib_.texcoords.push_back(x);
        attrib_.texcoords.push_back(y);
      } else if (tag == "mtllib") {
        std::string name;
        ss >> name;
        load_mtl(config.mtl_search_path + name, ids);
      } else if (tag == "usemtl") {
        std::string name;
        ss >> name;
        auto it = ids.find(name);
        cur = it == ids.end() ? -1 : it->second;
      } else if (tag == "f") {
        std::vector<index_t> poly;
        std::string c;
        while (ss >> c) {
          int idx[3] = {0, 0, 0};
          size_t pos = 0;
          for (int part = 0; part < 3; ++part) {
            const size_t slash = c.find('/', pos);
            const std::string tok = c.substr(pos, slash == std::string::npos ? std::string::npos : slash - pos);
            if (!tok.empty()) idx[part] = std::stoi(tok);
            if (slash == std::string::npos) break;
            pos = slash + 1;
          }
          index_t ix;
          ix.vertex_index = fix(idx[0], attrib_.vertices.size());
          ix.texcoord_index = idx[1] ? (idx[1] > 0 ? idx[1] - 1 : (int)attrib_.texcoords.size() / 2 + idx[1]) : -1;
          ix.normal_index = idx[2] ? fix(idx[2], attrib_.normals.size()) : -1;
          poly.push_back(ix);
        }
        for (size_t t = 1; t + 1 < poly.size(); ++t) {
          mesh_t& m = shapes_[0].mesh;
          m.indices.push_back(poly[0]);
          m.indices.push_back(poly[t]);
          m.indices.push_back(poly[t + 1]);
          m.num_face_vertices.push_back(3);
          m.material_ids.push_back(cur);
        }
      }
    }
    return true;
  }
  bool Valid() const { return error_.empty(); }
  const attrib_t& GetAttrib() const { return attrib_; }
  const std::vector<shape_t>& GetShapes() const { return shapes_; }
  const std::vector<material_t>& GetMaterials() const { return materials_; }
  const std::string& Warning() const { return warning_; }
  const std::string& Error() const { return error_; }
};
}  // namespace tinyobj
