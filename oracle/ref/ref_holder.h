// ref_holder.h — the scene object the checker entry points pass around
// (TEST INFRASTRUCTURE ONLY): a reference BVHRT created by CreateSceneRT.
#pragma once
#include <memory>

#include "MultiRenderer/BVH2Common.h"

struct LrtrHolder {
  std::shared_ptr<ISceneObject> obj;
  BVHRT* rt;
};
