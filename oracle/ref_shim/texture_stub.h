// TEST INFRASTRUCTURE ONLY (oracle).  Stands in for scene/texture.h, which
// needs SDL_gpu and stb_image: materials in the measured scenes carry no
// texture, so only the sentinel and a Texture with an Id() are needed.
#pragma once
#define TEXTURE_H
#include <SDL3/SDL.h>
static constexpr Uint32 kNoTexture = 0xFFFFFFFFu;
class Texture {
public:
    Uint32 Id() const { return 0; }
};
