// Reads a curve file through the drop-in header the way reference applications do
// (YarnBall::readFromPoly / readFromOBJ / readFromBCC with a glm-style mat4), then prints
// the vertex count, the number of joined vertices and the first position; a malformed file
// throws std::runtime_error with the reference's message.
#include <cstdio>
#include <cstring>
#include <stdexcept>

#include "yarnball/YarnBall.h"

int main(int argc, char** argv) {
    if (argc < 3) return 2;
    YarnBall::mat4 transform(1.f);
    transform[0][0] = transform[1][1] = transform[2][2] = 0.01f;
    try {
        YarnBall::Sim* sim = nullptr;
        const char* kind = argv[1];
        if (!std::strcmp(kind, "poly"))
            sim = YarnBall::readFromPoly(argv[2], 2e-3f, transform, false, true);
        else if (!std::strcmp(kind, "obj"))
            sim = YarnBall::readFromOBJ(argv[2], 2e-3f, transform, false, true);
        else
            sim = YarnBall::readFromBCC(argv[2], 2e-3f, transform, false, true);
        int joined = 0;
        for (int i = 0; i < sim->meta.numVerts; i++) joined += sim->verts[i].connectionIndex >= 0;
        std::printf("%d %d %.9g %.9g %.9g\n", sim->meta.numVerts, joined, sim->verts[0].pos.x, sim->verts[0].pos.y,
                    sim->verts[0].pos.z);
        delete sim;
    } catch (const std::runtime_error& e) {
        std::printf("error: %s\n", e.what());
        return 1;
    }
    return 0;
}
