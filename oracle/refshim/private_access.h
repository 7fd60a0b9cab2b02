// private_access.h - reads a private data member of a reference class without editing its header.
// TEST INFRASTRUCTURE ONLY.  An explicit template instantiation may name a private member
// ([temp.explicit]), and the friend function it defines hands the member pointer out, so the
// oracle can read the reference's own sketch arrays (CCSketchAlg::sketches, MCSketchAlg::sketches)
// to compare whole sketch sets byte for byte.
#pragma once

template <typename Tag, typename Tag::type Member>
struct GsRefPrivate {
  friend typename Tag::type gs_ref_member(Tag) { return Member; }
};
