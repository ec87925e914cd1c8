// The parts of tinyobjloader's interface that the reference's OBJ loader uses
// (app/Components/ObjectLoaders/OBJLoader.{hpp,cpp}), for the checker build only.
//
// TEST INFRASTRUCTURE ONLY.  tinyobjloader is an empty, unpinned submodule of the reference
// checkout, so its parser cannot be built here.  This header declares the same type and member
// names the loader's code reads (attrib_t, shape_t / mesh_t / index_t, material_t,
// MaterialStreamReader, LoadObj) so that OBJLoader::process and OBJLoader::fillScene compile
// unchanged.  LoadObj is defined by oracle/ref_driver.cpp: it ignores the streams and hands back a
// parse staged by the caller (the oracle's restatement of tinyobjloader's parser with triangulation),
// so the reference's own conversion code runs on it.
#ifndef MRT_ORACLE_TINY_OBJ_LOADER_H
#define MRT_ORACLE_TINY_OBJ_LOADER_H

#include <istream>
#include <map>
#include <string>
#include <vector>

namespace tinyobj {

typedef float real_t;

struct index_t {
    int vertex_index;
    int normal_index;
    int texcoord_index;
};

struct mesh_t {
    std::vector<index_t> indices;
    std::vector<unsigned int> num_face_vertices;   // vertices of each face (3 after triangulation)
    std::vector<int> material_ids;                 // per face, -1 without material
};

struct shape_t {
    std::string name;
    mesh_t mesh;
};

struct attrib_t {
    std::vector<real_t> vertices;    // 3 per vertex
    std::vector<real_t> normals;     // 3 per normal
    std::vector<real_t> texcoords;   // 2 per texture coordinate
    std::vector<real_t> colors;      // 3 per vertex (1, 1, 1 where the file gives none)
};

struct material_t {
    std::string name;
    real_t ambient[3];
    real_t diffuse[3];
    real_t specular[3];
    real_t transmittance[3];
    real_t emission[3];
    real_t shininess;
    real_t ior;
    real_t dissolve;
    int illum;
};

class MaterialReader {
public:
    virtual ~MaterialReader() = default;
};

class MaterialStreamReader : public MaterialReader {
public:
    explicit MaterialStreamReader(std::istream &in) : in_(in) {}

private:
    std::istream &in_;
};

bool LoadObj(attrib_t *attrib, std::vector<shape_t> *shapes, std::vector<material_t> *materials, std::string *warn,
             std::string *err, std::istream *in, MaterialReader *read_mat = nullptr, bool triangulate = true);

}  // namespace tinyobj

#endif
