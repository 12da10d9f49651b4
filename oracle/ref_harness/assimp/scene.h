// Minimal type-only stand-in for the assimp scene headers, written for the
// reference-harness build.  assimp is not installed on this machine; the
// reference only needs these names to compile its `import` asset branch
// (src/core/meta/scene.cu:27-135, src/core/primitive/mesh.cu:332-446).
// The importer below never returns a scene, so none of this is executed:
// meshes reach the reference through PolyMesh(vertices, normals, indices)
// (src/core/primitive/mesh.cu:404-433) from harness.cpp instead.
#pragma once
#include <cstddef>
#include <cstring>

struct aiVector3D {
    float x = 0, y = 0, z = 0;
};

struct aiMatrix4x4 {
    float a1 = 1, a2 = 0, a3 = 0, a4 = 0;
    float b1 = 0, b2 = 1, b3 = 0, b4 = 0;
    float c1 = 0, c2 = 0, c3 = 1, c4 = 0;
    float d1 = 0, d2 = 0, d3 = 0, d4 = 1;
    aiMatrix4x4 operator*(const aiMatrix4x4 &) const { return *this; }
    aiVector3D operator*(const aiVector3D &v) const { return v; }
};

struct aiString {
    char data[1024] = {0};
    const char *C_Str() const { return data; }
};

struct aiFace {
    unsigned mNumIndices = 0;
    unsigned *mIndices = nullptr;
};

struct aiMesh {
    unsigned mNumVertices = 0, mNumFaces = 0, mMaterialIndex = 0;
    aiVector3D *mVertices = nullptr, *mNormals = nullptr;
    aiFace *mFaces = nullptr;
    bool HasPositions() const { return false; }
    bool HasNormals() const { return false; }
    bool HasFaces() const { return false; }
};

struct aiNode {
    aiString mName;
    aiMatrix4x4 mTransformation;
    unsigned mNumMeshes = 0, mNumChildren = 0;
    unsigned *mMeshes = nullptr;
    aiNode **mChildren = nullptr;
    aiNode *FindNode(const aiString &) { return this; }
};

struct aiCamera {
    aiString mName;
    aiVector3D mPosition, mUp, mLookAt;
    float mHorizontalFOV = 0, mClipPlaneNear = 0, mClipPlaneFar = 0, mAspect = 0;
};

struct aiMaterial {
    template <typename... A> int Get(A &&...) const { return 0; }
};

#define AI_MATKEY_NAME "?mat.name", 0, 0
#define AI_SCENE_FLAGS_INCOMPLETE 0x1

struct aiScene {
    unsigned mFlags = 0;
    aiNode *mRootNode = nullptr;
    unsigned mNumMeshes = 0, mNumMaterials = 0, mNumCameras = 0;
    aiMesh **mMeshes = nullptr;
    aiMaterial **mMaterials = nullptr;
    aiCamera **mCameras = nullptr;
    bool HasCameras() const { return false; }
};
