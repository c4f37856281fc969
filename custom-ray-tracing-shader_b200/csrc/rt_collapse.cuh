// Collapse of the binary BVH into 8-wide compressed nodes (host and device).
//
// One job per wide node. A job is either a binary node (interior or leaf) or
// a range of primitives (a leaf too large for one node). For a binary node,
// the children start as its two children; the interior child with the largest
// surface area is opened (replaced by its two children) while the result
// still fits in eight slots, where a leaf of k <= 8 * group triangles needs
// ceil(k / group) slots (groups of up to `group` triangles, 1..3, each with
// its own box) and anything else one slot. Leaves that still do not fit become wide children of their own.
// Slots are assigned by ray octant (slot s holds the child nearest along
// direction signs s), and child boxes are quantised outward against the
// node's grid, checked with the same fused multiply-add the traversal uses.
#pragma once
#include "rt_build.cuh"

namespace rt {

RT_HD int imin(int a, int b) { return a < b ? a : b; }
RT_HD int imax(int a, int b) { return a > b ? a : b; }
RT_HD int portableAdd(int* p, int v) {
#ifdef __CUDA_ARCH__
    return atomicAdd(p, v);
#else
    int old = *p; *p += v; return old;
#endif
}
RT_HD void portableSet(int* p, int v) {
#ifdef __CUDA_ARCH__
    atomicExch(p, v);
#else
    *p = v;
#endif
}
RT_HD float collapseHalfArea(const float lo[3], const float hi[3]) {
    float x = fmaxf(0.0f, hi[0] - lo[0]), y = fmaxf(0.0f, hi[1] - lo[1]), z = fmaxf(0.0f, hi[2] - lo[2]);
    return x * y + x * z + y * z;
}
RT_HD void collapseGrow(float lo[3], float hi[3], const float olo[3], const float ohi[3]) {
    for (int a = 0; a < 3; a++) { lo[a] = fminf(lo[a], olo[a]); hi[a] = fmaxf(hi[a], ohi[a]); }
}

struct Job { int kind; int node; int first; int count; int wide; };  // kind 0 binary node, 1 primitive range
struct Kid { int kind; int node; int first; int count; float lo[3], hi[3]; };  // kind 0/1 wide child, 2 triangle group

// Slots a binary child needs: one for an interior node, ceil(k / group) for a
// leaf of k <= width * group triangles held inline, one for a larger leaf.
RT_HD int slotsOf(const BinNode& n, int group, int width) {
    if (n.count == 0) return 1;
    return n.count <= width * group ? (n.count + group - 1) / group : 1;
}

// A job's wide node before its storage is allocated: the children, their
// slots and boxes, and the triangles of each triangle group.
struct CollapsePlan {
    Kid kids[8];
    int nk, wide;
    int slotKid[8];
    int groupTris[8][3], groupCount[8];
    int nInterior, nTris;  // wide children (= next-level jobs) and packed triangles
    float nlo[3], nhi[3];
};

// Chooses up to eight children of job J's wide node, their boxes and slots,
// and the triangles of its triangle groups. width (4 or 8): most children
// per node; the node format keeps eight slots either way. primTri: the
// triangle of each primitive when primitives are triangle pieces (null:
// primitive p is triangle p).
RT_HD void planCollapse(Job J, const BinNode* bn, const int* order, const float4* plo, const float4* phi, int group,
                        int width, const int* primTri, CollapsePlan& P) {
    if (J.kind == 0 && bn[J.node].count > 0) { J.kind = 1; J.first = bn[J.node].first; J.count = bn[J.node].count; }
    P.wide = J.wide;
    Kid* kids = P.kids;
    int nk = 0;
    if (J.kind == 0) {
        int cand[8], nc = 2;
        bool asNode[8] = {false, false, false, false, false, false, false, false};
        cand[0] = bn[J.node].first; cand[1] = cand[0] + 1;
        for (;;) {
            int total = 0;
            for (int i = 0; i < nc; i++) total += slotsOf(bn[cand[i]], group, width);
            int best = -1; float bestArea = -1.0f;
            for (int i = 0; i < nc; i++) {
                const BinNode& c = bn[cand[i]];
                if (c.count != 0 || nc >= width) continue;
                int after = total - 1 + slotsOf(bn[c.first], group, width) + slotsOf(bn[c.first + 1], group, width);
                if (after > width) continue;
                float lo[3] = {c.low.x, c.low.y, c.low.z}, hi[3] = {c.high.x, c.high.y, c.high.z};
                float a = collapseHalfArea(lo, hi);
                if (a > bestArea) { bestArea = a; best = i; }
            }
            if (best < 0) break;
            int opened = cand[best];
            cand[best] = bn[opened].first;
            cand[nc++] = bn[opened].first + 1;
        }
        // Leaves that do not fit inline become wide children of their own.
        for (;;) {
            int total = 0;
            for (int i = 0; i < nc; i++) total += asNode[i] ? 1 : slotsOf(bn[cand[i]], group, width);
            if (total <= width) break;
            int pick = -1, most = 0;
            for (int i = 0; i < nc; i++) {
                const BinNode& c = bn[cand[i]];
                if (!asNode[i] && c.count > group && c.count > most) { most = c.count; pick = i; }
            }
            if (pick < 0) break;
            asNode[pick] = true;
        }
        for (int i = 0; i < nc && nk < width; i++) {
            const BinNode& c = bn[cand[i]];
            if (c.count == 0) {
                kids[nk++] = Kid{0, cand[i], 0, 0, {c.low.x, c.low.y, c.low.z}, {c.high.x, c.high.y, c.high.z}};
            } else if (asNode[i] || c.count > width * group) {
                kids[nk++] = Kid{1, -1, c.first, c.count, {c.low.x, c.low.y, c.low.z}, {c.high.x, c.high.y, c.high.z}};
            } else {
                for (int g = 0; g < c.count && nk < width; g += group)
                    kids[nk++] = Kid{2, -1, c.first + g, imin(group, c.count - g), {0, 0, 0}, {0, 0, 0}};
            }
        }
    } else if (J.count <= width * group) {
        for (int g = 0; g < J.count && nk < width; g += group)
            kids[nk++] = Kid{2, -1, J.first + g, imin(group, J.count - g), {0, 0, 0}, {0, 0, 0}};
    } else {
        int chunk = (J.count + width - 1) / width;
        for (int g = 0; g < J.count && nk < width; g += chunk) {
            int c = imin(chunk, J.count - g);
            kids[nk++] = Kid{c <= group ? 2 : 1, -1, J.first + g, c, {0, 0, 0}, {0, 0, 0}};
        }
    }
    // Boxes of primitive-range kids: union of padded primitive boxes.
    float nlo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, nhi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (int k = 0; k < nk; k++) {
        Kid& K = kids[k];
        if (K.kind != 0) {
            float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
            for (int i = 0; i < K.count; i++) {
                int p = order[K.first + i];
                float4 a = plo[p], b = phi[p];
                lo[0] = fminf(lo[0], a.x); lo[1] = fminf(lo[1], a.y); lo[2] = fminf(lo[2], a.z);
                hi[0] = fmaxf(hi[0], b.x); hi[1] = fmaxf(hi[1], b.y); hi[2] = fmaxf(hi[2], b.z);
            }
            for (int a = 0; a < 3; a++) { K.lo[a] = lo[a]; K.hi[a] = hi[a]; }
        }
        collapseGrow(nlo, nhi, K.lo, K.hi);
    }
    // Slot assignment: slot s holds the kid met first by rays whose direction
    // signs are s (bit 2 = x negative, bit 1 = y, bit 0 = z).
    int* slotKid = P.slotKid;
    for (int s = 0; s < 8; s++) slotKid[s] = -1;
    {
        float cn[3], ck[8][3];
        for (int a = 0; a < 3; a++) cn[a] = 0.5f * (nlo[a] + nhi[a]);
        for (int k = 0; k < nk; k++)
            for (int a = 0; a < 3; a++) ck[k][a] = 0.5f * (kids[k].lo[a] + kids[k].hi[a]) - cn[a];
        bool kidUsed[8] = {false, false, false, false, false, false, false, false};
        for (int round = 0; round < nk; round++) {
            float best = FLT_MAX; int bk = -1, bs = -1;
            for (int k = 0; k < nk; k++) {
                if (kidUsed[k]) continue;
                for (int s = 0; s < 8; s++) {
                    if (slotKid[s] >= 0) continue;
                    float c = ((s & 4) ? -ck[k][0] : ck[k][0]) + ((s & 2) ? -ck[k][1] : ck[k][1]) + ((s & 1) ? -ck[k][2] : ck[k][2]);
                    if (c < best) { best = c; bk = k; bs = s; }
                }
            }
            if (bk < 0) {  // non-finite costs: first free kid into the first free slot
                for (int k = 0; k < nk && bk < 0; k++) if (!kidUsed[k]) bk = k;
                for (int s = 0; s < 8 && bs < 0; s++) if (slotKid[s] < 0) bs = s;
            }
            kidUsed[bk] = true; slotKid[bs] = bk;
        }
    }
    // Triangles of each triangle group, once each: pieces of one triangle in
    // the same group would only repeat its test (the group's box covers them).
    int (*groupTris)[3] = P.groupTris;
    int* groupCount = P.groupCount;
    int nInterior = 0, nTris = 0;
    for (int k = 0; k < nk; k++) {
        groupCount[k] = 0;
        if (kids[k].kind != 2) { nInterior++; continue; }
        for (int i = 0; i < kids[k].count; i++) {
            const int prim = order[kids[k].first + i];
            const int tri = primTri ? primTri[prim] : prim;
            bool seen = false;
            for (int j = 0; j < groupCount[k]; j++) seen = seen || groupTris[k][j] == tri;
            if (!seen) groupTris[k][groupCount[k]++] = tri;
        }
        nTris += groupCount[k];
    }
    P.nk = nk;
    P.nInterior = nInterior;
    P.nTris = nTris;
    for (int a = 0; a < 3; a++) { P.nlo[a] = nlo[a]; P.nhi[a] = nhi[a]; }
}

// Writes a planned wide node whose storage has been allocated: wide children
// from childBase, packed triangles from triBase, next-level jobs from
// jobBase (nInterior of each). counters[3] receives an error code when an
// allocation passes its capacity.
RT_HD void emitCollapse(const CollapsePlan& P, int childBase, int triBase, int jobBase, const SceneTri* tris,
                        Job* nextJobs, WideNode* wide, float4* packed, int* counters, int wideCapacity,
                        int jobCapacity, int triCapacity) {
    const Kid* kids = P.kids;
    const int* slotKid = P.slotKid;
    const int (*groupTris)[3] = P.groupTris;
    const int* groupCount = P.groupCount;
    const float* nlo = P.nlo;
    const float* nhi = P.nhi;
    if (childBase + P.nInterior > wideCapacity || triBase + P.nTris > triCapacity) { portableSet(&counters[3], 3); return; }
    WideNode W;
    W.px = nlo[0]; W.py = nlo[1]; W.pz = nlo[2];
    float sc[3];
    unsigned char ebits[3];
    for (int a = 0; a < 3; a++) {
        float extent = nhi[a] - nlo[a];
        int ex = -126;
        if (extent > 0.0f) { frexpf(extent / 255.0f, &ex); }
        ex = imax(-126, imin(127, ex));
        ebits[a] = (unsigned char)(ex + 127);
        sc[a] = bitsToFloat((unsigned)ebits[a] << 23);
    }
    W.ex = ebits[0]; W.ey = ebits[1]; W.ez = ebits[2];
    W.imask = 0;
    W.childBase = (unsigned)childBase;
    W.triBase = (unsigned)triBase;
    int interiorSeen = 0, triOffset = 0;
    for (int s = 0; s < 8; s++) {
        int k = slotKid[s];
        if (k < 0) {
            W.meta[s] = 0;
            for (int a = 0; a < 3; a++) { W.qlo[a][s] = 0; W.qhi[a][s] = 0; }
            continue;
        }
        const Kid& K = kids[k];
        for (int a = 0; a < 3; a++) {
            float p = a == 0 ? W.px : (a == 1 ? W.py : W.pz);
            int ql = (int)floorf((K.lo[a] - p) / sc[a]);
            int qh = (int)ceilf((K.hi[a] - p) / sc[a]);
            ql = imax(0, imin(255, ql));
            qh = imax(0, imin(255, qh));
            while (ql > 0 && fmaRn((float)ql, sc[a], p) > K.lo[a]) ql--;
            while (qh < 255 && fmaRn((float)qh, sc[a], p) < K.hi[a]) qh++;
            W.qlo[a][s] = (unsigned char)ql;
            W.qhi[a][s] = (unsigned char)qh;
        }
        if (K.kind == 2) {
            const int count = groupCount[k];
            W.meta[s] = (unsigned char)((((1u << count) - 1u) << 5) | (unsigned)triOffset);
            for (int i = 0; i < count; i++) {
                const int p = groupTris[k][i];  // the triangle
                const SceneTri& t = tris[p];
                float4* dst = packed + (size_t)(triBase + triOffset + i) * 3;
                dst[0] = make_float4(t.origin.x, t.origin.y, t.origin.z, t.edge1.x);
                dst[1] = make_float4(t.edge1.y, t.edge1.z, t.edge2.x, t.edge2.y);
                dst[2] = make_float4(t.edge2.z, bitsToFloat(t.oneSided != 0 ? 1u : 0u), bitsToFloat((unsigned)p), 0.0f);
            }
            triOffset += count;
        } else {
            W.meta[s] = (unsigned char)(0x20u | (24u + (unsigned)s));
            W.imask |= (unsigned char)(1u << s);
            const int q = jobBase + interiorSeen;
            if (q >= jobCapacity) { portableSet(&counters[3], 4); interiorSeen++; continue; }
            nextJobs[q] = Job{K.kind == 0 ? 0 : 1, K.node, K.first, K.count, childBase + interiorSeen};
            interiorSeen++;
        }
    }
    wide[P.wide] = W;
}

// Builds wide node J.wide for one job: planCollapse, then allocation of its
// wide children, packed triangles and next-level jobs, then emitCollapse.
// counters: [0] wide nodes, [1] packed triangles, [2] next-level jobs,
// [3] error code. Host and device (atomics through portableAdd), so the
// collapse can be checked on the CPU. nextCount, when set, counts the
// next-level jobs in place of counters[2].
RT_HD void collapseJob(Job J, const BinNode* bn, const int* order, const float4* plo, const float4* phi,
                       const SceneTri* tris, Job* nextJobs, WideNode* wide, float4* packed, int* counters,
                       int wideCapacity, int jobCapacity, int triCapacity, int group, int width = 8,
                       const int* primTri = nullptr, int* nextCount = nullptr) {
    CollapsePlan P;
    planCollapse(J, bn, order, plo, phi, group, width, primTri, P);
    const int childBase = P.nInterior ? portableAdd(&counters[0], P.nInterior) : 0;
    const int triBase = P.nTris ? portableAdd(&counters[1], P.nTris) : 0;
    const int jobBase = P.nInterior ? portableAdd(nextCount ? nextCount : &counters[2], P.nInterior) : 0;
    emitCollapse(P, childBase, triBase, jobBase, tris, nextJobs, wide, packed, counters, wideCapacity, jobCapacity,
                 triCapacity);
}

}  // namespace rt
