/* ORACLE — test infrastructure only. Drives the reference's vendored MikkTSpace
 * (External/mikktspace/mikktspace.c, compiled from the reference tree into oracle/_ref/) the way the
 * reference's GenerateTangentSpace does (Core/Source/Utils/Math/TangentSpace.cpp:8-89): triangles of
 * an indexed mesh, per-corner results stored per vertex (the last corner naming a vertex wins). */
#include <mikktspace.h>
#include <stdint.h>

typedef struct
{
    const float *positions, *normals, *uvs;
    const uint32_t* indices;
    int triangles;
    float* tangents;
} mesh;

static int num_faces(const SMikkTSpaceContext* c) { return ((const mesh*)c->m_pUserData)->triangles; }
static int num_vertices(const SMikkTSpaceContext* c, int f) { (void)c; (void)f; return 3; }
static uint32_t vertex_of(const SMikkTSpaceContext* c, int f, int k) { return ((const mesh*)c->m_pUserData)->indices[f * 3 + k]; }

static void get_position(const SMikkTSpaceContext* c, float out[3], int f, int k)
{
    const float* p = ((const mesh*)c->m_pUserData)->positions + 3 * vertex_of(c, f, k);
    out[0] = p[0]; out[1] = p[1]; out[2] = p[2];
}
static void get_normal(const SMikkTSpaceContext* c, float out[3], int f, int k)
{
    const float* p = ((const mesh*)c->m_pUserData)->normals + 3 * vertex_of(c, f, k);
    out[0] = p[0]; out[1] = p[1]; out[2] = p[2];
}
static void get_uv(const SMikkTSpaceContext* c, float out[2], int f, int k)
{
    const float* p = ((const mesh*)c->m_pUserData)->uvs + 2 * vertex_of(c, f, k);
    out[0] = p[0]; out[1] = p[1];
}
static void set_basic(const SMikkTSpaceContext* c, const float t[3], float sign, int f, int k)
{
    float* o = ((mesh*)c->m_pUserData)->tangents + 4 * vertex_of(c, f, k);
    o[0] = t[0]; o[1] = t[1]; o[2] = t[2]; o[3] = sign;
}

int mikk_ref_tangents(const float* positions, const float* normals, const float* uvs, const uint32_t* indices, int triangles,
                      float* tangents)
{
    mesh m = {positions, normals, uvs, indices, triangles, tangents};
    SMikkTSpaceInterface iface = {0};
    iface.m_getNumFaces = num_faces;
    iface.m_getNumVerticesOfFace = num_vertices;
    iface.m_getPosition = get_position;
    iface.m_getNormal = get_normal;
    iface.m_getTexCoord = get_uv;
    iface.m_setTSpaceBasic = set_basic;
    SMikkTSpaceContext ctx = {0};
    ctx.m_pInterface = &iface;
    ctx.m_pUserData = &m;
    return genTangSpaceDefault(&ctx) ? 0 : 1;
}
