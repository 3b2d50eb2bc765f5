// Scene packing for the host-description calls (dvg_render, dvg_render_backward):
// one pass over the Python scene objects of dvg.scene (Scene, Shape, ShapeGroup,
// Path, Circle, Ellipse, Rect, paints) into the structure-of-arrays layout of
// dvg_scene_desc (include/dvg.h).  Python module `_dvgpack`; dvg.abi.pack_scene wraps
// it.  The arrays are the ones dvg.abi.pack_scene_python builds with plain Python, byte
// for byte (values go through the same double -> float32 rounding numpy applies).
#define PY_SSIZE_T_CLEAN
#include <Python.h>

#include <cstdint>
#include <cstring>
#include <vector>

namespace {

// the codes of include/dvg.h (dvg_shape_kind, dvg_paint_kind, path flags)
constexpr uint32_t SHAPE_CIRCLE = 0, SHAPE_RECT = 1, SHAPE_PATH = 2, SHAPE_ELLIPSE = 3;
constexpr uint32_t PAINT_SOLID = 1, PAINT_LINEAR = 2, PAINT_RADIAL = 3;
constexpr uint32_t PATH_CLOSED = 1, PATH_DISTANCE_APPROX = 2, PATH_HAS_THICKNESS = 4;

// Owned reference.
struct Ref {
    PyObject* o = nullptr;
    explicit Ref(PyObject* p = nullptr) : o(p) {}
    Ref(const Ref&) = delete;
    Ref& operator=(const Ref&) = delete;
    ~Ref() { Py_XDECREF(o); }
    PyObject* get() const { return o; }
    explicit operator bool() const { return o != nullptr; }
};

// Interned attribute names.
struct Names {
    PyObject *shapes, *groups, *geometry, *transform, *m, *stroke_width, *stroke_join, *stroke_cap,
        *stroke_miter_limit, *path, *points, *num_control_points, *thickness, *is_closed, *use_distance_approx,
        *center, *radius, *min, *max, *shape_indices, *fill_rule, *shape_to_canvas, *canvas_to_shape, *fill,
        *stroke, *r, *g, *b, *a, *start, *end, *stops, *offset, *color;
} N;

bool intern_names() {
#define I(x) (N.x = PyUnicode_InternFromString(#x)) != nullptr
    return I(shapes) && I(groups) && I(geometry) && I(transform) && I(m) && I(stroke_width) && I(stroke_join) &&
           I(stroke_cap) && I(stroke_miter_limit) && I(path) && I(points) && I(num_control_points) &&
           I(thickness) && I(is_closed) && I(use_distance_approx) && I(center) && I(radius) && I(min) && I(max) &&
           I(shape_indices) && I(fill_rule) && I(shape_to_canvas) && I(canvas_to_shape) && I(fill) && I(stroke) &&
           I(r) && I(g) && I(b) && I(a) && I(start) && I(end) && I(stops) && I(offset) && I(color);
#undef I
}

// The classes an isinstance test needs, and numpy.ascontiguousarray for matrices that
// are not float32 / float64 buffers.
struct Types {
    PyObject *path_geometry, *circle, *ellipse, *rect, *color, *linear, *radial, *as_f32;
};

PyObject* attr(PyObject* o, PyObject* name) { return PyObject_GetAttr(o, name); }

// float32(x) the way numpy converts a Python number: through a C double.
bool to_f32(PyObject* x, float* out) {
    const double d = PyFloat_AsDouble(x);
    if (d == -1.0 && PyErr_Occurred()) return false;
    *out = (float)d;
    return true;
}
bool attr_f32(PyObject* o, PyObject* name, float* out) {
    Ref v(attr(o, name));
    return v && to_f32(v.get(), out);
}
// int(x), then the range numpy's uint32 / int32 conversions accept.
bool to_int(PyObject* x, long long* out) {
    Ref v(PyNumber_Long(x));
    if (!v) return false;
    *out = PyLong_AsLongLong(v.get());
    return !(*out == -1 && PyErr_Occurred());
}
bool to_u32(PyObject* x, uint32_t* out) {
    long long v;
    if (!to_int(x, &v)) return false;
    if (v < 0 || v > 0xffffffffLL) {
        PyErr_SetString(PyExc_OverflowError, "value out of range for uint32");
        return false;
    }
    *out = (uint32_t)v;
    return true;
}
// item i of a sequence as float32
bool item_f32(PyObject* seq, Py_ssize_t i, float* out) {
    Ref v(PySequence_GetItem(seq, i));
    return v && to_f32(v.get(), out);
}
// Mat3.m: 9 float32 values, row-major.
bool matrix9(PyObject* mat, const Types& T, float* out) {
    Ref m(attr(mat, N.m));
    if (!m) return false;
    Py_buffer view;
    if (PyObject_GetBuffer(m.get(), &view, PyBUF_C_CONTIGUOUS | PyBUF_FORMAT) == 0) {
        const char* f = view.format ? view.format : "B";
        if (f[0] == '<' || f[0] == '=' || f[0] == '@') ++f;
        bool ok = false;
        if (f[0] == 'f' && f[1] == 0 && view.len == 9 * (Py_ssize_t)sizeof(float)) {
            std::memcpy(out, view.buf, 9 * sizeof(float));
            ok = true;
        } else if (f[0] == 'd' && f[1] == 0 && view.len == 9 * (Py_ssize_t)sizeof(double)) {
            const double* d = static_cast<const double*>(view.buf);
            for (int k = 0; k < 9; ++k) out[k] = (float)d[k];
            ok = true;
        }
        PyBuffer_Release(&view);
        if (ok) return true;
    } else {
        PyErr_Clear();
    }
    // anything else: numpy's own conversion, as the Python packer applies it
    Ref a(PyObject_CallOneArg(T.as_f32, m.get()));
    if (!a) return false;
    if (PyObject_GetBuffer(a.get(), &view, PyBUF_C_CONTIGUOUS) != 0) return false;
    const bool ok = view.len == 9 * (Py_ssize_t)sizeof(float);
    if (ok) std::memcpy(out, view.buf, 9 * sizeof(float));
    PyBuffer_Release(&view);
    if (!ok) PyErr_SetString(PyExc_ValueError, "a transform must have 9 entries");
    return ok;
}
// (v[0], v[1]) of a 2-vector attribute
bool vec2(PyObject* o, PyObject* name, float* x, float* y) {
    Ref v(attr(o, name));
    return v && item_f32(v.get(), 0, x) && item_f32(v.get(), 1, y);
}
int isinst(PyObject* o, PyObject* cls) { return PyObject_IsInstance(o, cls); }

template <typename T>
PyObject* bytes_of(const std::vector<T>& v) {
    return PyByteArray_FromStringAndSize(reinterpret_cast<const char*>(v.data()), (Py_ssize_t)(v.size() * sizeof(T)));
}

struct Packed {
    std::vector<uint32_t> kinds, joins, caps, ctrl_off, ctrl_cnt, pt_off, pt_cnt, flags, g_off, g_cnt, g_rule,
        p_kind, p_soff, p_scnt;
    std::vector<float> params, xforms, sw, miters, pts, thick, g_s2c, g_c2s, p_params, s_off, s_col;
    std::vector<uint8_t> ncp;
    std::vector<int64_t> g_ids;
    std::vector<int32_t> g_fill, g_stroke;
    bool any_thick = false;
};

bool pack_shape(PyObject* sh, const Types& T, Packed& P, std::vector<std::pair<size_t, std::vector<float>>>& th) {
    float xf[9];
    Ref tr(attr(sh, N.transform));
    if (!tr || !matrix9(tr.get(), T, xf)) return false;
    P.xforms.insert(P.xforms.end(), xf, xf + 9);
    float v;
    if (!attr_f32(sh, N.stroke_width, &v)) return false;
    P.sw.push_back(v);
    uint32_t u;
    {
        Ref j(attr(sh, N.stroke_join));
        if (!j || !to_u32(j.get(), &u)) return false;
        P.joins.push_back(u);
    }
    {
        Ref c(attr(sh, N.stroke_cap));
        if (!c || !to_u32(c.get(), &u)) return false;
        P.caps.push_back(u);
    }
    if (!attr_f32(sh, N.stroke_miter_limit, &v)) return false;
    P.miters.push_back(v);
    Ref g(attr(sh, N.geometry));
    if (!g) return false;
    int is = isinst(g.get(), T.path_geometry);
    if (is < 0) return false;
    if (is) {
        Ref p(attr(g.get(), N.path));
        if (!p) return false;
        Ref points(attr(p.get(), N.points)), ncps(attr(p.get(), N.num_control_points));
        if (!points || !ncps) return false;
        Ref pf(PySequence_Fast(points.get(), "path points must be a sequence"));
        Ref nf(PySequence_Fast(ncps.get(), "num_control_points must be a sequence"));
        if (!pf || !nf) return false;
        const Py_ssize_t npt = PySequence_Fast_GET_SIZE(pf.get()), nn = PySequence_Fast_GET_SIZE(nf.get());
        P.kinds.push_back(SHAPE_PATH);
        P.params.insert(P.params.end(), 4, 0.0f);
        P.ctrl_off.push_back((uint32_t)P.ncp.size());
        P.ctrl_cnt.push_back((uint32_t)nn);
        const size_t off = P.pts.size() / 2;
        P.pt_off.push_back((uint32_t)off);
        P.pt_cnt.push_back((uint32_t)npt);
        for (Py_ssize_t k = 0; k < nn; ++k) {
            long long c;
            if (!to_int(PySequence_Fast_GET_ITEM(nf.get(), k), &c)) return false;
            P.ncp.push_back((uint8_t)c);  // numpy int64 -> uint8 wraps the same way
        }
        for (Py_ssize_t k = 0; k < npt; ++k) {
            PyObject* q = PySequence_Fast_GET_ITEM(pf.get(), k);
            float x, y;
            if (PyTuple_CheckExact(q) && PyTuple_GET_SIZE(q) == 2) {
                if (!to_f32(PyTuple_GET_ITEM(q, 0), &x) || !to_f32(PyTuple_GET_ITEM(q, 1), &y)) return false;
            } else if (!item_f32(q, 0, &x) || !item_f32(q, 1, &y)) {
                return false;
            }
            P.pts.push_back(x);
            P.pts.push_back(y);
        }
        Ref closed(attr(p.get(), N.is_closed)), approx(attr(p.get(), N.use_distance_approx));
        if (!closed || !approx) return false;
        const int c = PyObject_IsTrue(closed.get()), a = PyObject_IsTrue(approx.get());
        if (c < 0 || a < 0) return false;
        uint32_t f = (c ? PATH_CLOSED : 0) | (a ? PATH_DISTANCE_APPROX : 0);
        Ref thick(attr(p.get(), N.thickness));
        if (!thick) return false;
        if (thick.get() != Py_None) {
            f |= PATH_HAS_THICKNESS;
            Ref tf(PySequence_Fast(thick.get(), "thickness must be a sequence"));
            if (!tf) return false;
            const Py_ssize_t nt = PySequence_Fast_GET_SIZE(tf.get());
            std::vector<float> t;
            for (Py_ssize_t k = 0; k < nt && k < npt; ++k) {
                float tv;
                if (!to_f32(PySequence_Fast_GET_ITEM(tf.get(), k), &tv)) return false;
                t.push_back(tv);
            }
            th.emplace_back(off, std::move(t));
            P.any_thick = true;
        }
        P.flags.push_back(f);
        return true;
    }
    P.ctrl_off.push_back(0);
    P.ctrl_cnt.push_back(0);
    P.pt_off.push_back(0);
    P.pt_cnt.push_back(0);
    P.flags.push_back(0);
    float q[4] = {0, 0, 0, 0};
    if ((is = isinst(g.get(), T.circle)) != 0) {
        if (is < 0 || !vec2(g.get(), N.center, &q[0], &q[1]) || !attr_f32(g.get(), N.radius, &q[2])) return false;
        P.kinds.push_back(SHAPE_CIRCLE);
    } else if ((is = isinst(g.get(), T.ellipse)) != 0) {
        if (is < 0 || !vec2(g.get(), N.center, &q[0], &q[1]) || !vec2(g.get(), N.radius, &q[2], &q[3])) return false;
        P.kinds.push_back(SHAPE_ELLIPSE);
    } else if ((is = isinst(g.get(), T.rect)) != 0) {
        if (is < 0 || !vec2(g.get(), N.min, &q[0], &q[1]) || !vec2(g.get(), N.max, &q[2], &q[3])) return false;
        P.kinds.push_back(SHAPE_RECT);
    } else {
        PyErr_Format(PyExc_TypeError, "unsupported geometry %R", (PyObject*)Py_TYPE(g.get()));
        return false;
    }
    P.params.insert(P.params.end(), q, q + 4);
    return true;
}

// One paint: kind, 4 parameters, stops.
bool pack_paint(PyObject* paint, const Types& T, Packed& P) {
    float q[4];
    uint32_t kind;
    PyObject* stops_name = nullptr;
    int is;
    if ((is = isinst(paint, T.color)) != 0) {
        if (is < 0 || !attr_f32(paint, N.r, &q[0]) || !attr_f32(paint, N.g, &q[1]) || !attr_f32(paint, N.b, &q[2]) ||
            !attr_f32(paint, N.a, &q[3]))
            return false;
        kind = PAINT_SOLID;
    } else if ((is = isinst(paint, T.linear)) != 0) {
        if (is < 0 || !vec2(paint, N.start, &q[0], &q[1]) || !vec2(paint, N.end, &q[2], &q[3])) return false;
        kind = PAINT_LINEAR;
        stops_name = N.stops;
    } else if ((is = isinst(paint, T.radial)) != 0) {
        if (is < 0 || !vec2(paint, N.center, &q[0], &q[1]) || !vec2(paint, N.radius, &q[2], &q[3])) return false;
        kind = PAINT_RADIAL;
        stops_name = N.stops;
    } else {
        PyErr_Format(PyExc_TypeError, "unsupported paint %R", (PyObject*)Py_TYPE(paint));
        return false;
    }
    P.p_kind.push_back(kind);
    P.p_params.insert(P.p_params.end(), q, q + 4);
    P.p_soff.push_back((uint32_t)P.s_off.size());
    if (!stops_name) {
        P.p_scnt.push_back(0);
        return true;
    }
    Ref st(attr(paint, stops_name));
    if (!st) return false;
    Ref sf(PySequence_Fast(st.get(), "stops must be a sequence"));
    if (!sf) return false;
    const Py_ssize_t ns = PySequence_Fast_GET_SIZE(sf.get());
    P.p_scnt.push_back((uint32_t)ns);
    for (Py_ssize_t k = 0; k < ns; ++k) {
        PyObject* s = PySequence_Fast_GET_ITEM(sf.get(), k);
        float o, c[4];
        if (!attr_f32(s, N.offset, &o)) return false;
        Ref col(attr(s, N.color));
        if (!col || !attr_f32(col.get(), N.r, &c[0]) || !attr_f32(col.get(), N.g, &c[1]) ||
            !attr_f32(col.get(), N.b, &c[2]) || !attr_f32(col.get(), N.a, &c[3]))
            return false;
        P.s_off.push_back(o);
        P.s_col.insert(P.s_col.end(), c, c + 4);
    }
    return true;
}

// pack(scene, (PathGeometry, Circle, Ellipse, Rect, Color, LinearGradient,
//              RadialGradient, as_float32)) -> (arrays: dict name -> bytearray,
//              any_thickness, paint_of: dict (group, "fill"|"stroke") -> paint index)
PyObject* pack(PyObject*, PyObject* args) {
    PyObject *scene, *types;
    if (!PyArg_ParseTuple(args, "OO!", &scene, &PyTuple_Type, &types)) return nullptr;
    if (PyTuple_GET_SIZE(types) != 8) {
        PyErr_SetString(PyExc_ValueError, "expected 8 type entries");
        return nullptr;
    }
    Types T{PyTuple_GET_ITEM(types, 0), PyTuple_GET_ITEM(types, 1), PyTuple_GET_ITEM(types, 2),
            PyTuple_GET_ITEM(types, 3), PyTuple_GET_ITEM(types, 4), PyTuple_GET_ITEM(types, 5),
            PyTuple_GET_ITEM(types, 6), PyTuple_GET_ITEM(types, 7)};
    Packed P;
    std::vector<std::pair<size_t, std::vector<float>>> th;
    Ref shapes(attr(scene, N.shapes));
    if (!shapes) return nullptr;
    Ref sf(PySequence_Fast(shapes.get(), "scene.shapes must be a sequence"));
    if (!sf) return nullptr;
    const Py_ssize_t ns = PySequence_Fast_GET_SIZE(sf.get());
    for (Py_ssize_t i = 0; i < ns; ++i)
        if (!pack_shape(PySequence_Fast_GET_ITEM(sf.get(), i), T, P, th)) return nullptr;
    P.thick.assign(P.pts.size() / 2, 0.0f);
    for (auto& t : th) std::copy(t.second.begin(), t.second.end(), P.thick.begin() + t.first);

    Ref paint_of(PyDict_New());
    if (!paint_of) return nullptr;
    Ref groups(attr(scene, N.groups));
    if (!groups) return nullptr;
    Ref gf(PySequence_Fast(groups.get(), "scene.groups must be a sequence"));
    if (!gf) return nullptr;
    const Py_ssize_t ng = PySequence_Fast_GET_SIZE(gf.get());
    for (Py_ssize_t gi = 0; gi < ng; ++gi) {
        PyObject* grp = PySequence_Fast_GET_ITEM(gf.get(), gi);
        Ref ids(attr(grp, N.shape_indices));
        if (!ids) return nullptr;
        Ref idf(PySequence_Fast(ids.get(), "shape_indices must be a sequence"));
        if (!idf) return nullptr;
        const Py_ssize_t nid = PySequence_Fast_GET_SIZE(idf.get());
        P.g_off.push_back((uint32_t)P.g_ids.size());
        P.g_cnt.push_back((uint32_t)nid);
        for (Py_ssize_t k = 0; k < nid; ++k) {
            long long v;
            if (!to_int(PySequence_Fast_GET_ITEM(idf.get(), k), &v)) return nullptr;
            P.g_ids.push_back(v);
        }
        uint32_t rule;
        Ref fr(attr(grp, N.fill_rule));
        if (!fr || !to_u32(fr.get(), &rule)) return nullptr;
        P.g_rule.push_back(rule);
        float m[9];
        Ref s2c(attr(grp, N.shape_to_canvas)), c2s(attr(grp, N.canvas_to_shape));
        if (!s2c || !c2s || !matrix9(s2c.get(), T, m)) return nullptr;
        P.g_s2c.insert(P.g_s2c.end(), m, m + 9);
        if (!matrix9(c2s.get(), T, m)) return nullptr;
        P.g_c2s.insert(P.g_c2s.end(), m, m + 9);
        // stroke first, then fill: the paint numbering of the Python packer
        for (int w = 0; w < 2; ++w) {
            Ref paint(attr(grp, w == 0 ? N.stroke : N.fill));
            if (!paint) return nullptr;
            std::vector<int32_t>& dst = w == 0 ? P.g_stroke : P.g_fill;
            if (paint.get() == Py_None) {
                dst.push_back(-1);
                continue;
            }
            const int32_t idx = (int32_t)P.p_kind.size();
            if (!pack_paint(paint.get(), T, P)) return nullptr;
            dst.push_back(idx);
            Ref key(Py_BuildValue("(ns)", gi, w == 0 ? "stroke" : "fill"));
            Ref val(PyLong_FromLong(idx));
            if (!key || !val || PyDict_SetItem(paint_of.get(), key.get(), val.get()) < 0) return nullptr;
        }
    }

    Ref arrays(PyDict_New());
    if (!arrays) return nullptr;
    auto put = [&](const char* name, PyObject* ba) -> bool {
        if (!ba) return false;
        const int r = PyDict_SetItemString(arrays.get(), name, ba);
        Py_DECREF(ba);
        return r == 0;
    };
    if (!put("kinds", bytes_of(P.kinds)) || !put("params", bytes_of(P.params)) || !put("xforms", bytes_of(P.xforms)) ||
        !put("sw", bytes_of(P.sw)) || !put("joins", bytes_of(P.joins)) || !put("caps", bytes_of(P.caps)) ||
        !put("miters", bytes_of(P.miters)) || !put("ctrl_off", bytes_of(P.ctrl_off)) ||
        !put("ctrl_cnt", bytes_of(P.ctrl_cnt)) || !put("pt_off", bytes_of(P.pt_off)) ||
        !put("pt_cnt", bytes_of(P.pt_cnt)) || !put("flags", bytes_of(P.flags)) || !put("ncp", bytes_of(P.ncp)) ||
        !put("pts", bytes_of(P.pts)) || !put("thick", bytes_of(P.thick)) || !put("g_off", bytes_of(P.g_off)) ||
        !put("g_cnt", bytes_of(P.g_cnt)) || !put("g_ids", bytes_of(P.g_ids)) || !put("g_rule", bytes_of(P.g_rule)) ||
        !put("g_s2c", bytes_of(P.g_s2c)) || !put("g_c2s", bytes_of(P.g_c2s)) || !put("g_fill", bytes_of(P.g_fill)) ||
        !put("g_stroke", bytes_of(P.g_stroke)) || !put("p_kind", bytes_of(P.p_kind)) ||
        !put("p_params", bytes_of(P.p_params)) || !put("p_soff", bytes_of(P.p_soff)) ||
        !put("p_scnt", bytes_of(P.p_scnt)) || !put("s_off", bytes_of(P.s_off)) || !put("s_col", bytes_of(P.s_col)))
        return nullptr;
    return Py_BuildValue("(OOO)", arrays.get(), P.any_thick ? Py_True : Py_False, paint_of.get());
}

PyMethodDef methods[] = {{"pack", pack, METH_VARARGS, "Pack a dvg.scene.Scene into dvg_scene_desc arrays."},
                         {nullptr, nullptr, 0, nullptr}};
PyModuleDef module = {PyModuleDef_HEAD_INIT, "_dvgpack", "Scene packing for the dvg host calls.", -1, methods,
                      nullptr, nullptr, nullptr, nullptr};

}  // namespace

PyMODINIT_FUNC PyInit__dvgpack(void) {
    if (!intern_names()) return nullptr;
    return PyModule_Create(&module);
}
