// Type-only stand-in (see scene.h in this folder): an importer that never
// loads anything, so the reference's `import` branch yields no meshes.
#pragma once
#include <string>
#include "scene.h"
namespace Assimp {
class Importer {
public:
    const aiScene *ReadFile(const std::string &, unsigned) { return nullptr; }
    void FreeScene() {}
};
}  // namespace Assimp
