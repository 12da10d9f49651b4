// Type-only stand-in (see scene.h in this folder): post-process flag names.
#pragma once
enum aiPostProcessSteps {
    aiProcess_CalcTangentSpace = 0x1,
    aiProcess_JoinIdenticalVertices = 0x2,
    aiProcess_Triangulate = 0x8,
    aiProcess_GenSmoothNormals = 0x40,
    aiProcess_FlipUVs = 0x800000,
};
