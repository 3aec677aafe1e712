#pragma once
// The iteration driver of the GraphOne API (reference: base/run.h:8-39):
// the functor picks its engine; the loop runs BeforeEngine -> Forward ->
// AfterEngine until the component or the frontier converges.

#include "GraphOne/utils/log.hpp"

namespace graph_one {

template <typename functor_t, typename comp_t, typename frontier_t>
void Run(comp_t& comp, frontier_t& frontier) {
    using engine_t = typename functor_t::template engine_type<functor_t, comp_t, frontier_t>;
    engine_t engine(comp, frontier);
    comp.Init();
    while (!comp.IsConvergent() && !frontier.IsConvergent()) {
        comp.BeforeEngine();
        frontier.BeforeEngine();
        engine.Forward();
        frontier.AfterEngine();
        comp.AfterEngine();
    }
    comp.Final();
}

}  // namespace graph_one
