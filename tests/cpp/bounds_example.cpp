// Sim::bounds() used the way the reference's callers use its Kitten::LBVH::aabb result
// (grow, pad, test, centre); prints whether every vertex lies inside the returned box and the
// padded box's volume.
#include <cstdio>

#include "yarnball/YarnBall.h"

using namespace YarnBall;

int main() {
    constexpr int numVerts = 64;
    auto sim = new YarnBall::Sim(numVerts);
    for (int i = 0; i < 32; i++) {
        vec3 pos = vec3(0.00002f * i * (i - 16) + 0.002f, -0.002f * i, 0);
        sim->verts[i].pos = pos;
        pos.x *= -1;
        sim->verts[i + 32].pos = pos;
    }
    sim->verts[0].invMass = sim->verts[32].invMass = sim->verts[63].invMass = 0;
    sim->verts[31].flags = 0;
    sim->configure();
    sim->upload();
    sim->advance(1 / 30.f);
    sim->download();
    auto box = sim->bounds();
    int inside = 0;
    for (int i = 0; i < numVerts; i++) inside += box.contains(sim->verts[i].pos);
    auto grown = box;
    grown.pad(0.01f);
    grown.absorb(vec3(1.f, 1.f, 1.f));
    const vec3 c = grown.center();
    printf("%d %d %d %.9g %.9g\n", inside, (int)grown.contains(box), (int)box.intersects(grown), grown.volume(), c[0]);
    delete sim;
    return 0;
}
