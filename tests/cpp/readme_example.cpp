// The README example of the reference (README.md:104-127) written against the drop-in
// header, unchanged apart from the include; prints the final positions of vertices 31 and 63.
#include <cstdio>

#include "yarnball/YarnBall.h"

using namespace YarnBall;

int main(int argc, char** argv) {
    const int frames = argc > 1 ? atoi(argv[1]) : 30;
    constexpr int numVerts = 64;
    auto sim = new YarnBall::Sim(numVerts);
    const float segLen = 0.002f;

    for (int i = 0; i < 32; i++) {
        vec3 pos = vec3(0.00002f * i * (i - 16) + segLen * 1, -segLen * i, 0);
        sim->verts[i].pos = pos;
        pos.x *= -1;
        sim->verts[i + 32].pos = pos;
    }

    sim->verts[0].invMass = sim->verts[32].invMass = sim->verts[63].invMass = 0;
    sim->verts[31].flags = 0;
    sim->meta.kCollision = 1e-7;
    sim->configure();
    sim->setKBend(1e-8);
    sim->setKStretch(2e-2);
    sim->maxH = 1e-3;
    sim->upload();

    for (int f = 0; f < frames; f++) sim->advance(1 / 30.f);
    sim->download();
    printf("%.9g %.9g %.9g\n", sim->verts[31].pos.x, sim->verts[31].pos.y, sim->verts[31].pos.z);
    printf("%.9g %.9g %.9g\n", sim->verts[63].pos.x, sim->verts[63].pos.y, sim->verts[63].pos.z);
    printf("steps %zu\n", sim->stepCount());
    delete sim;
    return 0;
}
