// Generated by gen_constants.py (mpmath, 2000-bit precision). Do not edit.
#pragma once
#include <cstdint>
namespace ionp {
constexpr double PI_2_1 = 0x1.921fb54442d18p+0;
constexpr double PI_2_2 = 0x1.1a62633145c07p-54;
constexpr double PI_2_3 = -0x1.f1976b7ed8fbcp-110;
constexpr double LN2_1 = 0x1.62e42fefa39efp-1;
constexpr double LN2_2 = 0x1.abc9e3b39803fp-56;
constexpr double LN2_3 = 0x1.7b57a079a1934p-111;
// 2/pi = 0.w0 w1 w2 ... (32 bits per word)
__host__ __device__ constexpr uint32_t two_over_pi_word(int i) {
    constexpr uint32_t W[48] = {0xA2F9836Eu, 0x4E441529u, 0xFC2757D1u, 0xF534DDC0u, 0xDB629599u, 0x3C439041u, 0xFE5163ABu, 0xDEBBC561u, 0xB7246E3Au, 0x424DD2E0u, 0x06492EEAu, 0x09D1921Cu, 0xFE1DEB1Cu, 0xB129A73Eu, 0xE88235F5u, 0x2EBB4484u, 0xE99C7026u, 0xB45F7E41u, 0x3991D639u, 0x835339F4u, 0x9C845F8Bu, 0xBDF9283Bu, 0x1FF897FFu, 0xDE05980Fu, 0xEF2F118Bu, 0x5A0A6D1Fu, 0x6D367ECFu, 0x27CB09B7u, 0x4F463F66u, 0x9E5FEA2Du, 0x7527BAC7u, 0xEBE5F17Bu, 0x3D0739F7u, 0x8A5292EAu, 0x6BFB5FB1u, 0x1F8D5D08u, 0x56033046u, 0xFC7B6BABu, 0xF0CFBC20u, 0x9AF4361Du, 0xA9E39161u, 0x5EE61B08u, 0x6599855Fu, 0x14A06840u, 0x8DFFD880u, 0x4D732731u, 0x06061556u, 0xCA73A8C9u};
    return (i >= 0 && i < 48) ? W[i] : 0u;
}
}  // namespace ionp
