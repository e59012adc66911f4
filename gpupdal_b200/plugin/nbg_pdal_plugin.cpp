// nbg_pdal_plugin.cpp — PDAL plugin packaging of the B200 path: one shared
// library registering filters.b200normal, filters.b200eigenvalues,
// filters.b200covariancefeatures, filters.b200approximatecoplanar,
// filters.b200estimaterank, filters.b200nndistance,
// filters.b200optimalneighborhood, filters.b200lof and filters.b200outlier.
// Each takes the options of the reference filter it stands for (the same
// names, defaults and checks, parsed by the library's stage layer), adds the
// same dimensions, and runs its per-point loop on the GPU through the C ABI
// (include/nbg_b200.h).
//
// Packaging follows the reference's plugin mechanism: PDAL loads
// libpdal_plugin_filter_<name>.so for a stage type filters.<name> found on
// PDAL_DRIVER_PATH and calls its extern "C" PF_initPlugin
// (pdal/PluginDirectory.cpp:70-100, pdal/PluginManager.cpp:316-347), the
// entry point CREATE_SHARED_STAGE writes (pdal/PluginHelper.hpp:60-66).  One
// library serves every stage: CMakeLists.txt installs it once per stage name
// (links to one file), and PF_initPlugin registers all of them.
//
// The view's X/Y/Z are doubles; the stage recovers the raw LAS integers
// (`scale` / `offset` options, default 0.01 / 0) and refuses a view whose
// coordinates are not exactly raw * scale + offset, instead of
// approximating.  GPU selection: option `device` (default 0).
#include <pdal/Filter.hpp>
#include <pdal/PluginHelper.hpp>
#include <pdal/PointView.hpp>

#include <map>
#include <memory>
#include <mutex>
#include <sstream>

#include "nbg_pdal_shim.hpp"

namespace pdal {

namespace {

// One library context per device for the process (contexts keep their grid
// and scratch caches between stages).
nbg_context* context_for(int device) {
    static std::mutex mu;
    static std::map<int, nbg_context*> ctx;
    std::lock_guard<std::mutex> lock(mu);
    auto it = ctx.find(device);
    if (it != ctx.end()) return it->second;
    nbg_context* c = nullptr;
    if (nbg_create(&c, device, 0) != NBG_OK) return nullptr;
    ctx[device] = c;
    return c;
}

}  // namespace

class B200NeighbourhoodFilter : public Filter {
public:
    explicit B200NeighbourhoodFilter(const nbg_pdal::StageSpec* spec) : m_spec(spec) {}
    std::string getName() const override { return m_spec->plugin_type; }

private:
    void addArgs(ProgramArgs& args) override {
        m_values.assign(m_spec->options.size(), std::string());
        m_args.clear();
        for (size_t i = 0; i < m_spec->options.size(); ++i)
            m_args.push_back(&args.add(m_spec->options[i], "see the reference filter", m_values[i]));
        args.add("scale", "LAS scale of X, Y, Z", m_scale, 0.01);
        args.add("offset", "LAS offset of X, Y, Z", m_offset, 0.0);
        args.add("device", "CUDA device", m_device, 0);
    }

    std::string optionsJson() const {
        std::vector<std::pair<std::string, std::string>> set;
        for (size_t i = 0; i < m_args.size(); ++i)
            if (m_args[i]->set()) set.emplace_back(m_spec->options[i], m_values[i]);
        return nbg_pdal::options_json(set);
    }

    void addDimensions(PointLayoutPtr layout) override {
        // the dimensions the reference filter registers
        nbg_filter* f = nullptr;
        char err[1024] = {0};
        if (nbg_filter_create(m_spec->base_type, optionsJson().c_str(), 1, 1, &f, err, sizeof err))
            throwError(err);
        char names[512] = {0};
        nbg_filter_dims(f, names, sizeof names);
        nbg_filter_free(f);
        m_dims.clear();
        std::stringstream ss(names);
        std::string name;
        while (std::getline(ss, name, ','))
            m_dims.push_back(layout->registerOrAssignDim(name, Dimension::Type::Double));
    }

    void prepared(PointTableRef table) override {
        // prepared()'s checks, with the input's OptimalKNN / OptimalRadius
        PointLayoutPtr layout(table.layout());
        m_hasKopt = layout->hasDim(Dimension::Id::OptimalKNN);
        m_hasRopt = layout->hasDim(Dimension::Id::OptimalRadius);
        nbg_filter* f = nullptr;
        char err[1024] = {0};
        if (nbg_filter_create(m_spec->base_type, optionsJson().c_str(), m_hasKopt, m_hasRopt, &f, err,
                              sizeof err))
            throwError(err);
        const std::string pre = nbg_filter_log(f);
        nbg_filter_free(f);
        if (!pre.empty()) log()->get(LogLevel::Warning) << pre;
    }

    void filter(PointView& view) override {
        const point_count_t n = view.size();
        if (!n) return;
        nbg_context* ctx = context_for(m_device);
        if (!ctx) throwError("no sm_100 GPU for this stage");
        std::vector<double> x(n), y(n), z(n), kopt, ropt;
        for (PointId i = 0; i < n; ++i) {
            x[i] = view.getFieldAs<double>(Dimension::Id::X, i);
            y[i] = view.getFieldAs<double>(Dimension::Id::Y, i);
            z[i] = view.getFieldAs<double>(Dimension::Id::Z, i);
        }
        if (m_hasKopt) {
            kopt.resize(n);
            for (PointId i = 0; i < n; ++i) kopt[i] = view.getFieldAs<double>(Dimension::Id::OptimalKNN, i);
        }
        if (m_hasRopt) {
            ropt.resize(n);
            for (PointId i = 0; i < n; ++i)
                ropt[i] = view.getFieldAs<double>(Dimension::Id::OptimalRadius, i);
        }
        // outputs start from the view's current values (rows the reference
        // skips keep them)
        std::vector<std::vector<double>> out(m_dims.size(), std::vector<double>(n));
        std::vector<double*> cols;
        for (size_t d = 0; d < m_dims.size(); ++d) {
            for (PointId i = 0; i < n; ++i) out[d][i] = view.getFieldAs<double>(m_dims[d], i);
            cols.push_back(out[d].data());
        }
        const double scale[3] = {m_scale, m_scale, m_scale}, offset[3] = {m_offset, m_offset, m_offset};
        std::string lg, err;
        const int rc = nbg_pdal::run_stage(ctx, m_spec->base_type, optionsJson(), x.data(), y.data(),
                                           z.data(), n, scale, offset,
                                           m_hasKopt ? kopt.data() : nullptr,
                                           m_hasRopt ? ropt.data() : nullptr, cols, lg, err);
        if (!lg.empty()) log()->get(LogLevel::Info) << lg;
        if (rc != NBG_OK) throwError(err);
        for (size_t d = 0; d < m_dims.size(); ++d)
            for (PointId i = 0; i < n; ++i) view.setField(m_dims[d], i, out[d][i]);
    }

    const nbg_pdal::StageSpec* m_spec;
    std::vector<std::string> m_values;
    std::vector<Arg*> m_args;
    std::vector<Dimension::Id> m_dims;
    double m_scale = 0.01, m_offset = 0.0;
    int m_device = 0;
    bool m_hasKopt = false, m_hasRopt = false;
};

// PluginManager constructs registered stages with `new C` (pdal/
// PluginManager.hpp:111-122): one default-constructible class per stage.
template <int I>
class B200Stage : public B200NeighbourhoodFilter {
public:
    B200Stage() : B200NeighbourhoodFilter(&nbg_pdal::stages()[I]) {}
};

template <int I>
void registerStages() {
    if constexpr (I > 0) registerStages<I - 1>();
    const nbg_pdal::StageSpec& s = nbg_pdal::stages()[I];
    PluginInfo info(s.plugin_type, std::string("B200 ") + s.base_type,
                    "https://pdal.org/stages/" + std::string(s.base_type) + ".html");
    PluginManager<Stage>::registerPlugin<B200Stage<I>>(info);
}

}  // namespace pdal

// What CREATE_SHARED_STAGE writes, for the library's nine stages.
extern "C" PDAL_EXPORT void PF_initPlugin() { pdal::registerStages<8>(); }
