// Stand-ins for the parts of Atrc's interface that the pt_cuda plugin
// (atrc_b200/csrc/plugin/pt_cuda_renderer.hpp) uses, so that the plugin can
// be compiled and run here without the reference's agz-utils dependency.
//
// Renderer keeps the reference's member layout and its async contract
// (src/tracer/include/agz/tracer/core/renderer.h:17-64,
//  src/tracer/src/core/core/renderer.cpp:5-38): stop_rendering_ and
// doing_rendering_ are adjacent one-byte std::atomic<bool>s, and
// render_async raises doing_rendering_ for the whole render.  A binding that
// read stop_rendering_ as a 4-byte int would see doing_rendering_ in it.
//
// ConfigGroup holds the JSON text that factory::config_to_json would print
// for the group (src/factory/src/utility/config_cvt.cpp:10-37: every value a
// string), plus its "type" for the creating context.
#pragma once

#include <atomic>
#include <functional>
#include <future>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <tuple>
#include <vector>

namespace agz::tracer {

using real = float;
template <class T> using RC = std::shared_ptr<T>;
template <class T> using Box = std::unique_ptr<T>;

struct Spectrum {
    real r = 0, g = 0, b = 0;
    Spectrum() = default;
    Spectrum(real r_, real g_, real b_) : r(r_), g(g_), b(b_) {}
};
struct Vec3 {
    real x = 0, y = 0, z = 0;
    Vec3() = default;
    Vec3(real x_, real y_, real z_) : x(x_), y(y_), z(z_) {}
};

template <class T> struct Image2D {
    int w = 0, h = 0;
    std::vector<T> texels;
    void initialize(int height, int width) {
        h = height;
        w = width;
        texels.assign(size_t(w) * h, T{});
    }
    T& operator()(int y, int x) { return texels[size_t(y) * w + x]; }
};

struct RenderTarget {
    Image2D<Spectrum> image;
    Image2D<Spectrum> albedo;
    Image2D<Vec3> normal;
    Image2D<real> denoise;
};

class Camera {
public:
    virtual ~Camera() = default;
};

class FilmFilter {
public:
    explicit FilmFilter(real r) : radius(r) {}
    virtual ~FilmFilter() = default;
    real radius;
};

class FilmFilterApplier {
public:
    FilmFilterApplier(int width, int height, RC<const FilmFilter> f) : w_(width), h_(height), f_(std::move(f)) {}
    int width() const noexcept { return w_; }
    int height() const noexcept { return h_; }
    real radius() const noexcept { return f_->radius; }

private:
    int w_, h_;
    RC<const FilmFilter> f_;
};

class Scene {
public:
    void set_camera(RC<const Camera> c) { cam_ = std::move(c); }
    const Camera* get_camera() const noexcept { return cam_.get(); }

private:
    RC<const Camera> cam_;
};

class RendererInteractor {
public:
    using PreviewFunc = std::function<Image2D<Spectrum>()>;
    virtual ~RendererInteractor() = default;
    virtual void progress(double percent, const PreviewFunc& get_image_preview) = 0;
    virtual void begin() = 0;
    virtual void end() = 0;
    virtual void new_stage() = 0;
    virtual void end_stage() = 0;
};

class Renderer {
protected:
    std::atomic<bool> stop_rendering_ = false;
    std::atomic<bool> doing_rendering_ = false;

    bool is_waitable_ = false;
    std::future<RenderTarget> async_thread_;

public:
    virtual ~Renderer() { stop_async(); }

    virtual RenderTarget render(FilmFilterApplier filter, Scene& scene, RendererInteractor& reporter) = 0;

    void render_async(FilmFilterApplier filter, Scene& scene, RendererInteractor& reporter) {
        stop_rendering_ = false;
        doing_rendering_ = true;
        async_thread_ = std::async(std::launch::async, [this, filter, &scene, &reporter]() {
            struct Done {
                std::atomic<bool>& f;
                ~Done() { f = false; }
            } done{doing_rendering_};
            return this->render(filter, scene, reporter);
        });
        is_waitable_ = true;
    }

    void stop_async() {
        if (is_waitable_) {
            stop_rendering_ = true;
            if (async_thread_.valid()) async_thread_.wait();
            stop_rendering_ = false;
            is_waitable_ = false;
        }
    }

    RenderTarget wait_async() {
        is_waitable_ = false;
        return async_thread_.get();
    }

    bool is_doing_rendering() const noexcept { return doing_rendering_; }
};

inline real& eps_storage() {
    static real e = real(3e-4);
    return e;
}
inline real EPS() noexcept { return eps_storage(); }
inline void set_eps(real e) noexcept { eps_storage() = e; }

struct ConfigGroup {
    std::string type;
    std::string json;
};
using Config = ConfigGroup;

namespace factory {

struct JSON {
    std::string text;
};
inline JSON config_to_json(const Config& c) { return {c.json}; }
inline std::string json_to_string(const JSON& j) { return j.text; }

class CreatingObjectException : public std::runtime_error {
public:
    using runtime_error::runtime_error;
};

class CreatingContext;

template <class T> class Creator {
public:
    virtual ~Creator() = default;
    virtual std::string name() const = 0;
    virtual RC<T> create(const ConfigGroup& params, CreatingContext& context) const = 0;
};

template <> class Creator<Camera> {
public:
    virtual ~Creator() = default;
    virtual std::string name() const = 0;
    virtual RC<Camera> create(const ConfigGroup& params, CreatingContext& context, real film_aspect) const = 0;
};

template <class T> class Factory {
public:
    void add_creator(Box<Creator<T>>&& c) {
        const std::string n = c->name();
        creators_[n] = std::move(c);
    }
    const Creator<T>* get_creator(const std::string& n) const {
        const auto it = creators_.find(n);
        return it == creators_.end() ? nullptr : it->second.get();
    }

private:
    std::map<std::string, Box<Creator<T>>> creators_;
};

class PathMapper {
public:
    virtual ~PathMapper() = default;
    virtual std::string map(const std::string& path) const = 0;
};

class CreatingContext {
public:
    CreatingContext();  // registers the stand-in creators (defined by the test)

    const PathMapper* path_mapper = nullptr;
    const ConfigGroup* reference_root = nullptr;

    template <class T> Factory<T>& factory() noexcept { return std::get<Factory<T>>(factories_); }
    template <class T> const Factory<T>& factory() const noexcept { return std::get<Factory<T>>(factories_); }

    template <class T, class... Args> RC<T> create(const ConfigGroup& params, Args&&... args) {
        const Creator<T>* c = factory<T>().get_creator(params.type);
        if (!c) throw CreatingObjectException("unknown creator type name: " + params.type);
        return c->create(params, *this, std::forward<Args>(args)...);
    }

private:
    std::tuple<Factory<Camera>, Factory<FilmFilter>, Factory<Renderer>> factories_;
};

}  // namespace factory
}  // namespace agz::tracer
