/*
 * yarnball_b200_scenes.h - seeded synthetic yarn geometry (host code, no GPU needed).
 *
 * No reference counterpart: the reference loads curves from files
 * (KittenEngine/YarnBall/io/reader.cpp:13-295).  These generators produce the random-walk
 * yarn piles used by the benchmark and tests, deterministically from a 64-bit seed.
 */
#ifndef YARNBALL_B200_SCENES_H
#define YARNBALL_B200_SCENES_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* numYarns random walks with vertsPerYarn[y] vertices each, segment length segLen, inside
 * [0,cube]^3, turning angle ~ N(0, turnSigma) per step, no two non-adjacent segments closer
 * than minDist.  posOut receives 3 floats per vertex, yarn after yarn.
 * Returns 0, -1 when a yarn could not be placed, -2 on invalid arguments. */
int yb_scene_random_walks(uint64_t seed, int32_t numYarns, const int32_t* vertsPerYarn, float segLen, float cube,
                          float turnSigma, float minDist, float* posOut);

/* numScenes independent scenes (scene s has yarnsPerScene[s] yarns; vertsPerYarn is the
 * concatenation of every scene's yarn lengths), each in its own [0,cube]^3, scene s seeded
 * from (seed, s); generated on `threads` host threads (0 = all).  Returns 0, -1-s when
 * scene s failed, -2 on invalid arguments. */
int yb_scene_random_walks_batch(uint64_t seed, int32_t numScenes, const int32_t* yarnsPerScene,
                                const int32_t* vertsPerYarn, float segLen, float cube, float turnSigma, float minDist,
                                float* posOut, int32_t threads);

/* The index-th output of xoshiro256** seeded by SplitMix64(seed) (for reproducibility checks). */
uint64_t yb_rng_u64(uint64_t seed, int32_t index);

#ifdef __cplusplus
}
#endif
#endif
